// otm_homo.cu -- Homogenization_H / MG_H / Grid_H replacement: hierarchy, solver driver and
// the homogenization entry points of the C ABI.
//
// One otm_homo handle owns its whole multigrid hierarchy on the device (no __constant__
// symbols, no global buffer registry), runs all its work on a private stream that is
// ordered after / before the caller's stream with events, and captures the iteration loop in
// a CUDA graph that is replayed until the device-side convergence flag is set.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "otm_common.cuh"
#include "otm_homo_impl.h"
#include "otm_solver_kernels.cuh"
#include "otm_template.h"

#include <cudaTypedefs.h>

namespace otm {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void set_error(const std::string& msg) { g_last_error = msg; }

otm_status cuda_fail(cudaError_t e, const char* what) {
  set_error(std::string(what) + ": " + cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return OTM_ERR_OUT_OF_MEMORY;
  return OTM_ERR_CUDA;
}

static otm_status invalid(const std::string& msg) {
  set_error(msg);
  return OTM_ERR_INVALID_ARGUMENT;
}

// ---------------------------------------------------------------------------------------
// Hierarchy construction (MG_H::build, homogenization/MG.cpp:13-44; coarsening rule
// Grid_H::coarse2, homogenization/grid.cpp:92-138, here always by 2 per axis).
// ---------------------------------------------------------------------------------------
static std::vector<Dims> level_dims(const int reso[3], int coarsest_max_dof) {
  std::vector<Dims> out;
  Dims d{reso[0], reso[1], reso[2]};
  while (true) {
    out.push_back(d);
    const bool can = d.nx % 2 == 0 && d.ny % 2 == 0 && d.nz % 2 == 0 && d.nx >= 8 && d.ny >= 8 && d.nz >= 8 &&
                     d.nv() > size_t(coarsest_max_dof);
    if (!can) break;
    d = Dims{d.nx / 2, d.ny / 2, d.nz / 2};
  }
  return out;
}

// Launch with programmatic stream serialization: the kernel may be scheduled while its
// predecessor drains and waits for it in pdl_wait() (every kernel launched this way starts with
// it). Inside a stream capture the dependency becomes a programmatic graph edge.
template <typename... KArgs, typename... Args>
static void launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t lc{};
  lc.gridDim = grid;
  lc.blockDim = block;
  lc.dynamicSmemBytes = smem;
  lc.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  cudaLaunchKernelEx(&lc, k, static_cast<KArgs>(args)...);
}

static constexpr int kMaxCoarsest = 1024;

// Galerkin product of one coarse level with 9 warps per 32 coarse vertices (3 fine offsets per
// warp). Measured on the 32^3 .. 4^3 levels of a 128^3 cell: 25 / 9.5 / 6.2 / 5.6 us, against
// 34 / 32 / 31 / 32 us with one thread per vertex (all 729 products of a vertex in one thread)
// and 87 / 16 / 12 / 4.6 us with one warp per fine offset.
constexpr int kGalSplit = 9;
static void launch_galerkin_coarse(Dims df, Dims dc, const float* stf, float* stc, int cb, cudaStream_t s) {
  using G = GalerkinShape<kGalSplit>;
  k_galerkin_coarse<kGalSplit><<<unsigned(ceil_div(dc.nv(), size_t(32 * G::kGroups))), G::kThreads, G::kSmem, s>>>(
      df, dc, stf, stc, cb);
}

static bool mixed_supported() { return true; }

otm_status Homo::alloc(void** p, size_t bytes) {
  cudaError_t e = pool ? cudaMallocFromPoolAsync(p, bytes, pool, stream) : cudaMalloc(p, bytes);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  allocations.push_back(*p);
  bytes_allocated += bytes;
  return OTM_OK;
}

Homo::~Homo() {
  if (side) {
    cudaStreamSynchronize(side);  // the coarse-operator chain may still use the buffers
    cudaStreamDestroy(side);
  }
  if (ev_fork) cudaEventDestroy(ev_fork);
  if (ev_coarse) cudaEventDestroy(ev_coarse);
  for (auto& g : graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  if (loop_exec) cudaGraphExecDestroy(loop_exec);
  if (stream && !external) cudaStreamDestroy(stream);
  if (ev_in) cudaEventDestroy(ev_in);
  if (ev_out) cudaEventDestroy(ev_out);
  for (int a = 0; a < 2; a++)
    for (int j = 0; j < kMaxChunk; j++)
      if (prof_ev[a][j]) cudaEventDestroy(prof_ev[a][j]);
  for (void* p : allocations) {
    if (pool)
      cudaFreeAsync(p, stream);
    else
      cudaFree(p);
  }
  if (sc_host) cudaFreeHost(sc_host);
}

otm_status Homo::build(const otm_config& c, cudaStream_t ext_stream, cudaMemPool_t ext_pool, bool external_mode) {
  cfg = c;
  external = external_mode;
  pool = ext_pool;
  for (int i = 0; i < 3; i++) {
    if (cfg.reso[i] < 2) return invalid("resolution must be >= 2 per axis");
    if (cfg.reso[i] > 1024) {
      set_error("axis resolution cannot exceed 1024");  // homogenization/grid.cpp:23-25
      return OTM_ERR_UNSUPPORTED;
    }
  }
  if (cfg.pre_smooth < 0 || cfg.post_smooth < 0 || cfg.pre_smooth + cfg.post_smooth == 0)
    return invalid("need at least one smoothing sweep");
  if (cfg.max_iter < 1) return invalid("max_iter must be >= 1");
  if (cfg.check_every < 1) cfg.check_every = 1;
  if (cfg.check_every > kMaxChunk) cfg.check_every = kMaxChunk;
  if (cfg.coarsest_max_dof < 8) cfg.coarsest_max_dof = 8;
  if (cfg.solver != OTM_SOLVER_PCG && cfg.solver != OTM_SOLVER_VCYCLE) return invalid("unknown solver");
  if (cfg.smoother != OTM_SMOOTHER_COLOR && cfg.smoother != OTM_SMOOTHER_TILED) return invalid("unknown smoother");
  if (cfg.precision < OTM_PRECISION_FP32 || cfg.precision > OTM_PRECISION_MIXED_FP16)
    return invalid("unknown precision");
  if (cfg.precision != OTM_PRECISION_FP32 && !mixed_supported()) {
    set_error("mixed-precision storage is not available in this build");
    return OTM_ERR_UNSUPPORTED;
  }
  if (cfg.solver == OTM_SOLVER_PCG && cfg.pre_smooth != cfg.post_smooth)
    return invalid("PCG needs a symmetric V-cycle (pre_smooth == post_smooth)");

  std::vector<Dims> dims = level_dims(cfg.reso, cfg.coarsest_max_dof);
  if (dims.back().nv() > size_t(kMaxCoarsest)) {
    set_error("coarsest level too large for the dense direct solve (aspect ratio too extreme)");
    return OTM_ERR_UNSUPPORTED;
  }
  // template matrices, element size 1/reso_x (homogenization/homogenization.cpp:211)
  template_matrices(1.0 / cfg.reso[0] / 2.0, &tm);
  if (tm.structure_error > 1e-9) {
    set_error("element matrix does not have the cube-Laplacian structure");
    return OTM_ERR_UNSUPPORTED;
  }
  op = FineOp{float(tm.c[0]), float(tm.c[1]), float(tm.c[2]), float(tm.c[3])};
  op0 = FineOp{1.f, float(tm.c[1] / tm.c[0]), float(tm.c[2] / tm.c[0]), float(tm.c[3] / tm.c[0])};
  mixed = cfg.precision != OTM_PRECISION_FP32;
  face = !tm.face_zero;
  for (int j = 0; j < 8; j++)
    for (int cc = 0; cc < 3; cc++) {
      ef.disp[j][cc] = float(tm.disp[j][cc]);
      ef.feMu[j][cc] = float(tm.feMu[j][cc]);
    }

  if (external) {
    stream = ext_stream;
  } else {
    OTM_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    OTM_CUDA(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
    OTM_CUDA(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
  }
  // a handle of its own gets the side stream; the server's handles (external mode) already run
  // many requests side by side on their lanes, and a second stream per lane would exceed the
  // device's hardware queues and serialise unrelated lanes
  if (!external) {
    OTM_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    OTM_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    OTM_CUDA(cudaEventCreateWithFlags(&ev_coarse, cudaEventDisableTiming));
  }
  if (cfg.profile)
    for (int a = 0; a < 2; a++)
      for (int j = 0; j < kMaxChunk; j++) OTM_CUDA(cudaEventCreate(&prof_ev[a][j]));

  lv.resize(dims.size());
  for (size_t l = 0; l < dims.size(); l++) {
    Level& L = lv[l];
    L.d = dims[l];
    const size_t nv = L.d.nv();
    // the mixed form keeps the fine-level correction and residual in 16-bit buffers instead
    const bool fp32_fine = !(mixed && l == 0 && dims.size() > 1);
    if (fp32_fine) {
      OTM_TRY(alloc((void**)&L.u, 3 * nv * sizeof(float)));
      OTM_TRY(alloc((void**)&L.r, 3 * nv * sizeof(float)));
      OTM_CUDA(cudaMemsetAsync(L.u, 0, 3 * nv * sizeof(float), stream));
      OTM_CUDA(cudaMemsetAsync(L.r, 0, 3 * nv * sizeof(float), stream));
    }
    OTM_TRY(alloc((void**)&L.f, 3 * nv * sizeof(float)));
    OTM_CUDA(cudaMemsetAsync(L.f, 0, 3 * nv * sizeof(float), stream));
    if (l > 0 || dims.size() == 1) OTM_TRY(alloc((void**)&L.st, 27 * nv * sizeof(float)));
  }
  const size_t nv = lv[0].d.nv();
  OTM_TRY(alloc((void**)&ks, nv * sizeof(float)));
  OTM_TRY(alloc((void**)&kraw, nv * sizeof(float)));
  OTM_TRY(alloc((void**)&b, 3 * nv * sizeof(float)));
  OTM_TRY(alloc((void**)&x, 3 * nv * sizeof(float)));
  OTM_CUDA(cudaMemsetAsync(x, 0, 3 * nv * sizeof(float), stream));
  if (mixed) {
    if (lv.size() == 1) {
      set_error("mixed precision needs at least two multigrid levels");
      return OTM_ERR_UNSUPPORTED;
    }
    OTM_TRY(alloc((void**)&x64, 3 * nv * sizeof(double)));
    OTM_TRY(alloc(&k16, nv * 2));
    OTM_TRY(alloc(&u16, 3 * nv * 2));
    OTM_TRY(alloc(&r16, 3 * nv * 2));
    OTM_CUDA(cudaMemsetAsync(x64, 0, 3 * nv * sizeof(double), stream));
    OTM_CUDA(cudaMemsetAsync(u16, 0, 3 * nv * 2, stream));
  }
  OTM_TRY(alloc((void**)&p, 3 * nv * sizeof(float)));
  OTM_TRY(alloc((void**)&q, 3 * nv * sizeof(float)));
  OTM_CUDA(cudaMemsetAsync(p, 0, 3 * nv * sizeof(float), stream));
  nc = int(lv.back().d.nv());
  OTM_TRY(alloc((void**)&Ainv, size_t(nc) * nc * sizeof(double)));
  OTM_TRY(alloc((void**)&table, 64 * 27 * sizeof(float)));
  OTM_TRY(alloc((void**)&sc, sizeof(SolveScalars)));
  OTM_TRY(alloc((void**)&partials, size_t(kMaxPartials) * 16 * sizeof(double)));
  OTM_TRY(alloc((void**)&means, 8 * sizeof(double)));
  OTM_TRY(alloc((void**)&flags, 4 * sizeof(int)));
  OTM_CUDA(cudaMemsetAsync(sc, 0, sizeof(SolveScalars), stream));
  OTM_CUDA(cudaMemsetAsync(flags, 0, 4 * sizeof(int), stream));
  // pinned block: solve scalars, then the level-1 Galerkin table (uploaded from pinned memory
  // so the copy never waits for the stream)
  OTM_CUDA(cudaMallocHost((void**)&sc_host, sizeof(SolveScalars) + 64 * 27 * sizeof(float) + 4 * sizeof(int)));
  std::memset(sc_host, 0, sizeof(SolveScalars));
  float* tab = (float*)(sc_host + 1);
  flags_host = (int*)(tab + 64 * 27);
  galerkin_level1_table(tm, tab);
  OTM_CUDA(cudaMemcpyAsync(table, tab, 64 * 27 * sizeof(float), cudaMemcpyHostToDevice, stream));
  if (!external) OTM_CUDA(cudaStreamSynchronize(stream));
  // small levels (<= 16^3 unknowns) and the coarsest solve run in one single-CTA kernel
  {
    const int L = int(lv.size());
    int t = -1;
    for (int l = 1; l < L; l++)
      if (lv[l].d.nv() <= size_t(kTailMaxNv)) {
        t = l;
        break;
      }
    if (t > 0 && t < L - 1 && L - t <= kTailMaxLevels) {
      size_t floats = 0;
      for (int l = t; l < L; l++) floats += 9 * lv[l].d.nv();
      if (floats * sizeof(float) <= size_t(kMaxDynSmem)) {
        tail_l = t;
        tail_smem = floats * sizeof(float);
        OTM_CUDA(cudaFuncSetAttribute(k_vcycle_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem));
      }
    }
  }
  // the levels from the first with <= 32^3 unknowns (cluster_cycle 3) or <= 16^3 (cluster_cycle 2)
  // and the coarsest solve in one thread-block-cluster launch; cluster_cycle 1 takes <= 16^3 when
  // the level above that is smoothed by the coarse tile kernels (a sweep there is one launch, and
  // the cluster's passes cost a cluster barrier per half sweep), else <= 32^3
  if (cfg.cluster_cycle) {
    const int L = int(lv.size());
    size_t cl_max = cfg.cluster_cycle == 2 ? size_t(kClMaxNv / 8) : size_t(kClMaxNv);
    if (cfg.cluster_cycle == 1) {
      const bool ctiles = cfg.smoother == OTM_SMOOTHER_TILED && cfg.solver == OTM_SOLVER_PCG && cfg.pre_smooth > 1 &&
                          cfg.post_smooth > 1;
      for (int l = 2; l < L - 1; l++)
        if (lv[l].d.nv() <= size_t(kClMaxNv / 8)) {
          if (ctiles && lv[l - 1].d.nv() <= size_t(kClMaxNv) && ctile_fits(lv[l - 1].d)) cl_max = kClMaxNv / 8;
          break;
        }
    }
    int t = -1;
    for (int l = 1; l < L - 1; l++)
      if (lv[l].d.nv() <= cl_max) {
        t = l;
        break;
      }
    if (t > 0) {
      std::vector<Dims> dims;
      for (int l = t; l < L; l++) dims.push_back(lv[l].d);
      ClDesc cd{};
      const size_t bytes = cl_plan(dims.data(), int(dims.size()), &cd);
      if (bytes > 0 &&
          cudaFuncSetAttribute(k_vcycle_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem) ==
              cudaSuccess &&
          cudaFuncSetAttribute(k_vcycle_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
        cudaLaunchConfig_t lc{};
        lc.gridDim = dim3(kCl);
        lc.blockDim = dim3(kClThreads);
        lc.dynamicSmemBytes = bytes;
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, (void*)k_vcycle_cluster, &lc) == cudaSuccess && ncl >= 1) {
          cd.pre = cfg.pre_smooth;
          cd.post = cfg.post_smooth;
          for (int i = 0; i < cd.nlev; i++) {
            cd.lv[i].st = lv[t + i].st;
            cd.lv[i].rg = lv[t + i].r;
          }
          cd.Ainv = Ainv;
          cl_tables(&cd, cl_tab_host);
          OTM_TRY(alloc((void**)&cl_tab, cl_tab_host.size() * sizeof(int)));
          OTM_CUDA(cudaMemcpyAsync(cl_tab, cl_tab_host.data(), cl_tab_host.size() * sizeof(int),
                                   cudaMemcpyHostToDevice, stream));
          cd.tab_g = cl_tab;
          cl_desc = cd;
          cluster_l = t;
          cluster_smem = bytes;
        }
      }
      cudaGetLastError();  // a refused attribute or occupancy query leaves no error behind
    }
  }
  // the tile-staged fine smoother: cube elements (no face couplings), every axis a multiple of the
  // tile, a coarser level to correct from, at least two sweeps in each leg (consecutive sweeps move
  // the tile faces by half a tile; with one sweep per leg both legs would keep the faces of one
  // tiling, and the 128^3 design loop at V(1,1) ran 354 against 389 iterations/s with the colour
  // passes), and the PCG solver. Block
  // Jacobi across the tile faces leaves the mode that is constant inside each tile and alternates in
  // sign from tile to tile almost undamped (a smoother factor near -1): preconditioned CG is not
  // affected by that (the preconditioner stays symmetric positive definite), but stationary V-cycles
  // would stall on it, so they keep the global colour passes.
  if (cfg.smoother == OTM_SMOOTHER_TILED && cfg.solver == OTM_SOLVER_PCG && !face && lv.size() > 1 &&
      tile_fits(lv[0].d) && cfg.pre_smooth > 1 && cfg.post_smooth > 1) {
    OTM_TRY(tile_attributes());
    // the second buffer of the sweep ping-pong (the fine correction's storage type)
    OTM_TRY(alloc(&u2, 3 * lv[0].d.nv() * (mixed ? 2 : sizeof(float))));
    // per-tile partial sums of the tiled direction update (p . q)
    OTM_TRY(alloc((void**)&tile_partials, size_t(tile_count(lv[0].d)) * 3 * sizeof(double)));
    tiled = true;
  }
  // coarse levels smoothed by the tile kernels: the levels between the fine level and the cluster
  // or single-CTA cycle (or the coarsest level) whose axes are multiples of the coarse tile, under
  // the same conditions as the fine level's tiles
  if (cfg.smoother == OTM_SMOOTHER_TILED && cfg.solver == OTM_SOLVER_PCG && cfg.pre_smooth > 1 && cfg.post_smooth > 1) {
    const int L = int(lv.size());
    int last = L - 1;  // first level not smoothed by regular passes
    if (cluster_l > 0) last = std::min(last, cluster_l);
    if (tail_l > 0) last = std::min(last, tail_l);
    for (int l = 1; l < last; l++) {
      if (!ctile_fits(lv[l].d)) continue;
      OTM_TRY(alloc((void**)&lv[l].u2, 3 * lv[l].d.nv() * sizeof(float)));
      lv[l].ctiled = true;
    }
  }
  stats.levels = int(lv.size());
  stats.cluster_level = cluster_l;
  stats.smoother = tiled ? OTM_SMOOTHER_TILED : OTM_SMOOTHER_COLOR;
  stats.coarsest_reso[0] = lv.back().d.nx;
  stats.coarsest_reso[1] = lv.back().d.ny;
  stats.coarsest_reso[2] = lv.back().d.nz;
  return OTM_OK;
}

// Dynamic shared memory of the tile kernels (a per-function attribute of the current device; set
// at every build, which is cheap) and the TMA map of the fine right-hand side: a 4-D tensor
// {nx, ny, nz, 3 cases} of FP32 read in boxes {8, 8, 4, 3}, eight per tile.
otm_status Homo::tile_attributes() {
  const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  OTM_CUDA(cudaFuncSetAttribute(k_tile_apply_dot, a, int(kTileSmemResid)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_sweep<kFromZero, float, float>, a, int(kTileSmemSweep)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_sweep<kFromU, float, float>, a, int(kTileSmemSweep)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_sweep<kFromUProlong, float, float>, a, int(kTileSmemProlong)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_resid<float, float>, a, int(kTileSmemResid)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_sweep<kFromZero, __nv_bfloat16, __nv_bfloat16>, a, int(kTileSmemSweep)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_sweep<kFromU, __nv_bfloat16, __nv_bfloat16>, a, int(kTileSmemSweep)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_sweep<kFromUProlong, __nv_bfloat16, __nv_bfloat16>, a, int(kTileSmemProlong)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_resid<__nv_bfloat16, __nv_bfloat16>, a, int(kTileSmemResid)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_sweep<kFromZero, __half, __half>, a, int(kTileSmemSweep)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_sweep<kFromU, __half, __half>, a, int(kTileSmemSweep)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_sweep<kFromUProlong, __half, __half>, a, int(kTileSmemProlong)));
  OTM_CUDA(cudaFuncSetAttribute(k_tile_resid<__half, __half>, a, int(kTileSmemResid)));
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    OTM_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !fn) {
      set_error("cuTensorMapEncodeTiled is not available from the driver");
      return OTM_ERR_UNSUPPORTED;
    }
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const Dims d = lv[0].d;
  const cuuint64_t dims[4] = {cuuint64_t(d.nx), cuuint64_t(d.ny), cuuint64_t(d.nz), 3};
  const cuuint64_t strides[3] = {cuuint64_t(d.nx) * 4, cuuint64_t(d.nx) * d.ny * 4, cuuint64_t(d.nv()) * 4};
  const cuuint32_t box[4] = {cuuint32_t(kFBX), cuuint32_t(kFBY), cuuint32_t(kFBZ), 3};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = encode(&fmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, lv[0].f, dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed for the fine right-hand side");
    return OTM_ERR_CUDA;
  }
  return OTM_OK;
}

otm_status Homo::join_coarse() {
  if (!coarse_pending) return OTM_OK;
  OTM_CUDA(cudaStreamWaitEvent(stream, ev_coarse, 0));
  coarse_pending = false;
  return OTM_OK;
}

otm_status Homo::enter() {
  if (external) return OTM_OK;
  OTM_CUDA(cudaEventRecord(ev_in, user_stream));
  OTM_CUDA(cudaStreamWaitEvent(stream, ev_in, 0));
  return OTM_OK;
}

otm_status Homo::leave() {
  if (external) return OTM_OK;
  OTM_CUDA(cudaEventRecord(ev_out, stream));
  OTM_CUDA(cudaStreamWaitEvent(user_stream, ev_out, 0));
  return OTM_OK;
}

// ---------------------------------------------------------------------------------------
// update: import k, Galerkin stencils of every coarse level, dense coarsest inverse
// (Homogenization_H::update, homogenization/homogenization.cpp:76-81; MG_H::updateStencils,
// homogenization/MG.cpp:144-151).
// ---------------------------------------------------------------------------------------
otm_status Homo::update(const float* kin, int pitchT) {
  const Dims d0 = lv[0].d;
  if (!kin) return invalid("k pointer is NULL");
  if (pitchT <= 0) pitchT = d0.nx;
  if (pitchT < d0.nx) return invalid("pitchT smaller than the x resolution");
  OTM_TRY(enter());
  OTM_TRY(join_coarse());  // a previous field's coarse chain may still read ks
  const size_t nv = d0.nv();
  OTM_CUDA(cudaMemsetAsync(flags, 0, 2 * sizeof(int), stream));  // import / coarsest status of this field
  k_import<<<ceil_div(nv, kBlock), kBlock, 0, stream>>>(d0, kin, pitchT, cfg.power_penal, ks, kraw, flags);
  OTM_CHECK_LAUNCH("k_import");
  launched(1);
  return update_operators();
}

// update() from a density field: the density chain's forward pass (filter, SIMP map) writes the
// conductivities straight into this handle (no k field, no import pass), then the operators are
// built as in update().
otm_status Homo::update_density(const DensityArgs& a) {
  const Dims d0 = lv[0].d;
  OTM_TRY(enter());
  OTM_TRY(join_coarse());
  OTM_CUDA(cudaMemsetAsync(flags, 0, 2 * sizeof(int), stream));
  OTM_TRY(density_forward_import(d0, a.rho, a.rho_pitchT, a.rho_f, a.dk, a.wsum, a.weight_type, a.radius, a.periodic,
                                 a.p, a.k0, a.kmin, kraw, ks, cfg.power_penal, flags, stream));
  launched(1);
  return update_operators();
}

// Galerkin stencils of every coarse level and the dense coarsest inverse for the imported ks (the
// coarse chain on a side stream), then leave().
otm_status Homo::update_operators() {
  const Dims d0 = lv[0].d;
  const size_t nv = d0.nv();
  const int L = int(lv.size());
  const unsigned int* kmax_bits = (const unsigned int*)(flags + 2);
  if (mixed) {
    OTM_CUDA(cudaMemsetAsync(flags + 2, 0, sizeof(int), stream));
    k_kmax<<<reduce_blocks(nv), kBlock, 0, stream>>>(nv, ks, (unsigned int*)(flags + 2));
    if (cfg.precision == OTM_PRECISION_MIXED_BF16)
      k_to16<__nv_bfloat16><<<ceil_div(nv, kBlock), kBlock, 0, stream>>>(nv, ks, kmax_bits, (__nv_bfloat16*)k16);
    else
      k_to16<__half><<<ceil_div(nv, kBlock), kBlock, 0, stream>>>(nv, ks, kmax_bits, (__half*)k16);
    OTM_CHECK_LAUNCH("k_to16");
    launched(2);
  }
  // the coarse chain on the side stream (if any), after the import (and the 16-bit copies)
  cudaStream_t cs = side ? side : stream;
  if (side) {
    OTM_CUDA(cudaEventRecord(ev_fork, stream));
    OTM_CUDA(cudaStreamWaitEvent(side, ev_fork, 0));
  }
  for (int l = 1; l < L; l++) {
    const bool cb = (l < L - 1);  // smoothed levels use the colour-blocked stencil order
    const size_t nvc = lv[l].d.nv();
    if (l == 1)
      k_galerkin_fine<<<ceil_div(nvc, kBlock), kBlock, 0, cs>>>(lv[0].d, lv[1].d, ks, table, lv[1].st, cb,
                                                                mixed ? kmax_bits : nullptr, op.c0);
    else
      launch_galerkin_coarse(lv[l - 1].d, lv[l].d, lv[l - 1].st, lv[l].st, cb, cs);
    OTM_CHECK_LAUNCH("galerkin");
    launched(1);
  }
  if (L == 1) {
    k_fine_stencil<<<ceil_div(nv, kBlock), kBlock, 0, cs>>>(d0, ks, op, lv[0].st);
    OTM_CHECK_LAUNCH("k_fine_stencil");
    launched(1);
  }
  {
    const size_t abytes = size_t(nc) * nc * sizeof(double);
    const int use_smem = abytes <= size_t(kMaxDynSmem);
    if (use_smem)
      OTM_CUDA(cudaFuncSetAttribute(k_coarsest_build, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem));
    k_coarsest_build<<<1, 1024, use_smem ? abytes : 0, cs>>>(lv.back().d, lv.back().st, Ainv, flags + 1,
                                                              use_smem);
  }
  OTM_CHECK_LAUNCH("k_coarsest_build");
  launched(1);
  if (side) {
    OTM_CUDA(cudaEventRecord(ev_coarse, side));
    coarse_pending = true;
  }
  updated = true;
  solved = false;
  return leave();
}

// ---------------------------------------------------------------------------------------
// V-cycle and iteration (MG_H::v_cycle, homogenization/MG.cpp:46-71).
// ---------------------------------------------------------------------------------------
// Fine-level operations of the mixed form on 16-bit storage T: what = 0 colour pass,
// 1 residual, 2 restriction to level 1, 3 prolongation from level 1, 4 zero fill and first
// colour-pair pass.
template <typename T>
void Homo::fine_ops16(int what, int color) {
  Level& L = lv[0];
  const size_t nv = L.d.nv();
  const T* kk = (const T*)k16;
  T* u = (T*)u16;
  T* r = (T*)r16;
  const double* fs = sc->fscale;
  switch (what) {
    case 0:  // color is a colour pair (0..3) unless face entries are present
      if (face)
        k_gs_fine<true, 3, T, T><<<ceil_div(nv >> 3, kBlock), kBlock, 0, stream>>>(L.d, color, kk, op0, u, L.f, sc, fs);
      else
        k_gs_fine_pair<3, T, T><<<ceil_div(nv >> 3, kBlock), kBlock, 0, stream>>>(L.d, color, kk, op0, u, L.f, sc, fs);
      break;
    case 1:
      if (face)
        k_resid_fine<true, 3, T, T><<<ceil_div(nv, kBlock), kBlock, 0, stream>>>(L.d, kk, op0, u, L.f, r, sc, fs);
      else
        k_resid_fine<false, 3, T, T><<<ceil_div(nv, kBlock), kBlock, 0, stream>>>(L.d, kk, op0, u, L.f, r, sc, fs);
      break;
    case 2:
      k_restrict<3, T><<<ceil_div(lv[1].d.nv(), kBlock), kBlock, 0, stream>>>(L.d, lv[1].d, r, lv[1].f, sc,
                                                                            nullptr, size_t(0));
      break;
    case 4:  // zero fill + first colour-pair pass (paired colours only)
      k_gs_fine_pair_first<3, T, T><<<ceil_div(nv >> 3, kBlock), kBlock, 0, stream>>>(L.d, kk, op0, u, L.f, sc, fs);
      break;
    default:
      k_prolong8<3, T><<<ceil_div(lv[1].d.nv(), kBlock), kBlock, 0, stream>>>(L.d, lv[1].d, lv[1].u, u, sc);
      break;
  }
  launched(1);
}

// The zero fill of level l's correction and the first colour pass of its first sweep.
void Homo::gs_first(int l) {
  Level& L = lv[l];
  const size_t nsub = L.d.nv() >> 3;
  if (l == 0 && mixed) {
    if (cfg.precision == OTM_PRECISION_MIXED_BF16)
      fine_ops16<__nv_bfloat16>(4, 0);
    else
      fine_ops16<__half>(4, 0);
    return;
  }
  if (l == 0)
    launch_pdl(k_gs_fine_pair_first<3, float, float>, dim3(ceil_div(nsub, kBlock)), dim3(kBlock), 0, stream, L.d,
               (const float*)ks, op, L.u, (const float*)L.f, (const SolveScalars*)sc, (const double*)nullptr);
  else
    launch_pdl(k_gs_coarse_first<3>, dim3(ceil_div(nsub, kBlock)), dim3(kBlock), 0, stream, L.d, (const float*)L.st,
               L.u, (const float*)L.f, (const SolveScalars*)sc);
  launched(1);
}

void Homo::gs(int l, int color) {
  Level& L = lv[l];
  const size_t nsub = L.d.nv() >> 3;
  if (l == 0 && mixed) {
    if (cfg.precision == OTM_PRECISION_MIXED_BF16)
      fine_ops16<__nv_bfloat16>(0, color);
    else
      fine_ops16<__half>(0, color);
    return;
  }
  if (l == 0) {
    if (face)
      launch_pdl(k_gs_fine<true, 3>, dim3(ceil_div(nsub, kBlock)), dim3(kBlock), 0, stream, L.d, color, ks, op, L.u, L.f,
                 sc, nullptr);
    else  // color is a colour pair (0..3)
      launch_pdl(k_gs_fine_pair<3>, dim3(ceil_div(nsub, kBlock)), dim3(kBlock), 0, stream, L.d, color, ks, op, L.u,
                 L.f, sc, nullptr);
  } else {
    launch_pdl(k_gs_coarse<3>, dim3(ceil_div(nsub, kBlock)), dim3(kBlock), 0, stream, L.d, color, L.st, L.u, L.f, sc);
  }
  launched(1);
}

void Homo::vcycle(int l) {
  Level& L = lv[l];
  const size_t nv = L.d.nv();
  if (l == cluster_l) {
    ClDesc cd = cl_desc;
    cd.f_in = L.f;
    cd.u_out = L.u;
    cd.pre = cfg.pre_smooth;
    cd.post = cfg.post_smooth;
    launch_pdl(k_vcycle_cluster, dim3(kCl), dim3(kClThreads), cluster_smem, stream, cd, sc);
    launched(1);
    return;
  }
  if (l == tail_l) {
    TailDesc td{};
    td.nlev = int(lv.size()) - l;
    td.pre = cfg.pre_smooth;
    td.post = cfg.post_smooth;
    td.nc = nc;
    int off = 0;
    for (int i = 0; i < td.nlev; i++) {
      td.lv[i].d = lv[l + i].d;
      td.lv[i].st = lv[l + i].st;
      td.lv[i].off = off;
      off += int(9 * lv[l + i].d.nv());
    }
    td.f_in = L.f;
    td.u_out = L.u;
    td.Ainv = Ainv;
    launch_pdl(k_vcycle_tail, dim3(1), dim3(kTailThreads), tail_smem, stream, td, sc);
    launched(1);
    return;
  }
  if (l == int(lv.size()) - 1) {
    launch_pdl(k_coarsest_solve, dim3(1), dim3(std::min(1024, std::max(32, (nc + 31) / 32 * 32))), 3 * nc * sizeof(double), stream, 
        nc, Ainv, L.f, L.u, sc);
    launched(1);
    return;
  }
  if (l == 0 && tiled) {
    const double* fs = mixed ? (const double*)sc->fscale : nullptr;
    if (!mixed)
      vcycle_fine_tiled<float, float>(ks, L.u, L.r, op, fs);
    else if (cfg.precision == OTM_PRECISION_MIXED_BF16)
      vcycle_fine_tiled<__nv_bfloat16, __nv_bfloat16>((const __nv_bfloat16*)k16, (__nv_bfloat16*)u16,
                                                      (__nv_bfloat16*)r16, op0, fs);
    else
      vcycle_fine_tiled<__half, __half>((const __half*)k16, (__half*)u16, (__half*)r16, op0, fs);
    return;
  }
  if (l > 0 && L.ctiled) {
    vcycle_coarse_tiled(l);
    return;
  }
  const bool m16 = (l == 0 && mixed);
  const bool bf = cfg.precision == OTM_PRECISION_MIXED_BF16;
  // the first pass of the first sweep starts from u = 0: one kernel writes the zero fill and the
  // pass's values (not for the fine level with face entries, whose colours are not paired)
  const bool first_fused = cfg.pre_smooth > 0 && !(l == 0 && face);
  if (!first_fused) {
    if (m16)
      cudaMemsetAsync(u16, 0, 3 * nv * 2, stream);
    else
      cudaMemsetAsync(L.u, 0, 3 * nv * sizeof(float), stream);
  }
  // the fine level of the cube element sweeps colour pairs (4 launches), coarse levels 8 colours
  const int passes = (l == 0 && !face) ? 4 : 8;
  for (int s = 0; s < cfg.pre_smooth; s++)
    for (int c = 0; c < passes; c++) {
      if (s == 0 && c == 0 && first_fused)
        gs_first(l);
      else
        gs(l, c);
    }
  Level& C = lv[l + 1];
  if (m16) {
    if (bf) {
      fine_ops16<__nv_bfloat16>(1, 0);
      fine_ops16<__nv_bfloat16>(2, 0);
    } else {
      fine_ops16<__half>(1, 0);
      fine_ops16<__half>(2, 0);
    }
  } else {
    if (l == 0) {
      if (face)
        launch_pdl(k_resid_fine<true, 3>, dim3(ceil_div(nv, kBlock)), dim3(kBlock), 0, stream, L.d, ks, op, L.u, L.f,
                   L.r, sc, nullptr);
      else
        launch_pdl(k_resid_fine<false, 3>, dim3(ceil_div(nv, kBlock)), dim3(kBlock), 0, stream, L.d, ks, op, L.u, L.f,
                   L.r, sc, nullptr);
    } else {
      launch_pdl(k_resid_coarse<3>, dim3(ceil_div(nv, kBlock)), dim3(kBlock), 0, stream, L.d, L.st, L.u, L.f, L.r, sc);
    }
    launch_pdl(k_restrict<3>, dim3(ceil_div(C.d.nv(), kBlock)), dim3(kBlock), 0, stream, L.d, C.d, L.r, C.f, sc,
               st_prefetch(l + 1), st_prefetch_bytes(l + 1));
    launched(2);  // residual + restriction
  }
  if (l == 0 && join_in_cycle) {
    // the coarse levels need the operators of the side stream's chain from here on
    if (coarse_pending) cudaStreamWaitEvent(stream, ev_coarse, 0);
    coarse_pending = false;
    join_in_cycle = false;
  }
  vcycle(l + 1);
  if (m16) {
    if (bf)
      fine_ops16<__nv_bfloat16>(3, 0);
    else
      fine_ops16<__half>(3, 0);
  } else {
    launch_pdl(k_prolong8<3, float>, dim3(ceil_div(C.d.nv(), kBlock)), dim3(kBlock), 0, stream, L.d, C.d,
               (const float*)C.u, L.u, (const SolveScalars*)sc);
    launched(1);
  }
  for (int s = 0; s < cfg.post_smooth; s++) {
    // the profiled sweep: the first post-smoothing sweep of the fine level (plain colour passes)
    const bool timed = cfg.profile && l == 0 && s == 0 && prof_slot >= 0;
    // inside a stream capture only an "external" event record becomes a graph node
    const unsigned int evflag = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    if (timed) cudaEventRecordWithFlags(prof_ev[0][prof_slot], stream, evflag);
    for (int c = passes - 1; c >= 0; c--) gs(l, c);
    if (timed) cudaEventRecordWithFlags(prof_ev[1][prof_slot], stream, evflag);
  }
}

// The fine level of the V-cycle with the tile kernels. Pre-smoothing: one launch per sweep,
// starting from u = 0, tilings 0, 1, 0, ... (ping-pong between u and u2); the residual of its
// result into r and the restriction; the coarse cycle; post-smoothing with the tilings mirrored
// (the last sweep on tiling 0), the first sweep adding the prolongation of the coarse correction,
// the last one writing the V-cycle's result (the preconditioned residual) into r.
template <typename KT, typename VT>
void Homo::vcycle_fine_tiled(const KT* k, VT* u, VT* r, const FineOp& fop, const double* fs) {
  Level& L = lv[0];
  Level& C = lv[1];
  const unsigned nt = tile_count(L.d);
  VT* buf[2] = {u, (VT*)u2};
  const int npre = cfg.pre_smooth, npost = cfg.post_smooth;
  launch_pdl(k_tile_sweep<kFromZero, KT, VT>, dim3(nt), dim3(kSmoothThreads), kTileSmemSweep, stream, fmap, L.d, C.d,
             k, fop, (const VT*)nullptr, (const float*)nullptr, buf[0], fs, 0, 0, sc);
  for (int s = 1; s < npre; s++)
    launch_pdl(k_tile_sweep<kFromU, KT, VT>, dim3(nt), dim3(kSmoothThreads), kTileSmemSweep, stream, fmap, L.d, C.d,
               k, fop, (const VT*)buf[(s - 1) & 1], (const float*)nullptr, buf[s & 1], fs, s & 1, 0, sc);
  VT* pre = buf[(npre - 1) & 1];
  launch_pdl(k_tile_resid<KT, VT>, dim3(nt), dim3(kResidThreads), kTileSmemResid, stream, fmap, L.d, k, fop,
             (const VT*)pre, r, fs, sc);
  launch_pdl(k_restrict<3, VT>, dim3(ceil_div(C.d.nv(), kBlock)), dim3(kBlock), 0, stream, L.d, C.d, (const VT*)r,
             C.f, (const SolveScalars*)sc, st_prefetch(1), st_prefetch_bytes(1));
  launched(npre + 2);
  if (join_in_cycle) {
    // the coarse levels need the operators of the side stream's chain from here on
    if (coarse_pending) cudaStreamWaitEvent(stream, ev_coarse, 0);
    coarse_pending = false;
    join_in_cycle = false;
  }
  vcycle(1);
  // the profiled region: the post-smoothing leg (post_smooth single-sweep launches)
  const bool timed = cfg.profile && prof_slot >= 0;
  const unsigned int evflag = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
  if (timed) cudaEventRecordWithFlags(prof_ev[0][prof_slot], stream, evflag);
  VT* in = pre;
  for (int s = 0; s < npost; s++) {
    VT* out = (s == npost - 1) ? r : (in == buf[0] ? buf[1] : buf[0]);
    const int shift = (npost - 1 - s) & 1;
    if (s == 0)
      launch_pdl(k_tile_sweep<kFromUProlong, KT, VT>, dim3(nt), dim3(kSmoothThreads), kTileSmemProlong, stream, fmap,
                 L.d, C.d, k, fop, (const VT*)in, (const float*)C.u, out, fs, shift, 1, sc);
    else
      launch_pdl(k_tile_sweep<kFromU, KT, VT>, dim3(nt), dim3(kSmoothThreads), kTileSmemSweep, stream, fmap, L.d,
                 C.d, k, fop, (const VT*)in, (const float*)nullptr, out, fs, shift, 1, sc);
    in = out;
  }
  if (timed) cudaEventRecordWithFlags(prof_ev[1][prof_slot], stream, evflag);
  launched(npost);
}

// A coarse level of the V-cycle with the tile kernels: pre-smoothing sweeps from u = 0 on the
// tilings 0, 1, 0, ..., ending in u2; the residual into r and its restriction; the coarser cycle;
// post-smoothing on the mirrored tilings, the first sweep adding the prolongation of the coarser
// correction, the last writing the level's result into u (which the finer level prolongs).
void Homo::vcycle_coarse_tiled(int l) {
  Level& L = lv[l];
  Level& C = lv[l + 1];
  const unsigned nt = ctile_count(L.d);
  const int npre = cfg.pre_smooth, npost = cfg.post_smooth;
  const float* none = nullptr;
  float* in = nullptr;
  for (int s = 0; s < npre; s++) {
    float* out = ((npre - 1 - s) % 2 == 0) ? L.u2 : L.u;
    if (s == 0)
      launch_pdl(k_ctile_sweep<kFromZero>, dim3(nt), dim3(kCThreads), kCTileSmem, stream, L.d, C.d,
                 (const float*)L.st, none, none, out, (const float*)L.f, 0, 0, (const SolveScalars*)sc);
    else
      launch_pdl(k_ctile_sweep<kFromU>, dim3(nt), dim3(kCThreads), kCTileSmem, stream, L.d, C.d, (const float*)L.st,
                 (const float*)in, none, out, (const float*)L.f, s & 1, 0, (const SolveScalars*)sc);
    in = out;
  }
  const float* pre = in;
  launch_pdl(k_resid_coarse<3>, dim3(ceil_div(L.d.nv(), kBlock)), dim3(kBlock), 0, stream, L.d, (const float*)L.st, pre,
             (const float*)L.f, L.r, (const SolveScalars*)sc);
  launch_pdl(k_restrict<3, float>, dim3(ceil_div(C.d.nv(), kBlock)), dim3(kBlock), 0, stream, L.d, C.d,
             (const float*)L.r, C.f, (const SolveScalars*)sc, st_prefetch(l + 1), st_prefetch_bytes(l + 1));
  launched(npre + 2);
  vcycle(l + 1);
  const float* pin = pre;
  for (int s = 0; s < npost; s++) {
    float* out = (s == npost - 1) ? L.u : (pin == L.r ? L.u2 : L.r);
    const int shift = (npost - 1 - s) & 1;
    if (s == 0)
      launch_pdl(k_ctile_sweep<kFromUProlong>, dim3(nt), dim3(kCThreads), kCTileSmemProlong, stream, L.d, C.d,
                 (const float*)L.st, pin, (const float*)C.u, out, (const float*)L.f, shift, 1, (const SolveScalars*)sc);
    else
      launch_pdl(k_ctile_sweep<kFromU>, dim3(nt), dim3(kCThreads), kCTileSmem, stream, L.d, C.d, (const float*)L.st,
                 pin, none, out, (const float*)L.f, shift, 1, (const SolveScalars*)sc);
    pin = out;
  }
  launched(npost);
}

// rho = r . z, then p = (z - zbar) + beta p, q = A p and alpha (z in its storage type VT).
template <typename VT>
void Homo::pcg_direction(const VT* z, const float* r, bool face, int nb) {
  const Dims d0 = lv[0].d;
  const size_t nv = d0.nv();
  launch_pdl(k_dot_rz<VT>, dim3(nb), dim3(kBlock), 0, stream, nv, r, z, partials, sc);
  // FP32 with the tile smoother: the tiled direction update (z's neighbours from shared memory)
  if (tiled && std::is_same<VT, float>::value && !face)
    launch_pdl(k_tile_apply_dot, dim3(tile_count(d0)), dim3(kResidThreads), kTileSmemResid, stream, d0,
               (const float*)ks, op, (const float*)z, p, q, tile_partials, sc);
  else if (face)
    launch_pdl(k_update_p_apply_dot<true, VT>, dim3(nb), dim3(kBlock), 0, stream, d0, ks, op, z, p, q, partials, sc);
  else
    launch_pdl(k_update_p_apply_dot<false, VT>, dim3(nb), dim3(kBlock), 0, stream, d0, ks, op, z, p, q, partials, sc);
}

void Homo::iteration(int j) {
  prof_slot = j;
  const Dims d0 = lv[0].d;
  const size_t nv = d0.nv();
  const int nb = reduce_blocks(nv);
  float* r = lv[0].f;  // Krylov residual is the V-cycle's level-0 right-hand side
  void* zv = fine_z();  // and the V-cycle's level-0 result is the preconditioned residual
  float* z = (float*)zv;
  if (mixed && cfg.solver == OTM_SOLVER_PCG) {
    // PCG with the 16-bit V-cycle as preconditioner, the solution in FP64 and exact FP64
    // residual replacements (k_update_x64r requests them, k_resid64 mode 2 performs them)
    const unsigned int* kmax_bits = (const unsigned int*)(flags + 2);
    vcycle(0);
    // z = xscale_c * u16 is read in place by the two kernels that use it
    if (cfg.precision == OTM_PRECISION_MIXED_BF16)
      pcg_direction((const __nv_bfloat16*)zv, r, face, nb);
    else
      pcg_direction((const __half*)zv, r, face, nb);
    launch_pdl(k_update_x64r, dim3(nb), dim3(kBlock), 0, stream, nv, x64, r, p, q, partials, sc, kmax_bits, op.c0,
               cfg.max_iter);
    if (face)
      launch_pdl(k_resid64<true>, dim3(nb), dim3(kBlock), 0, stream, d0, ks, op, x64, b, r, partials, sc, kmax_bits,
                 cfg.max_iter, 2);
    else
      launch_pdl(k_resid64<false>, dim3(nb), dim3(kBlock), 0, stream, d0, ks, op, x64, b, r, partials, sc, kmax_bits,
                 cfg.max_iter, 2);
    launched(4);
  } else if (mixed) {
    // FP64 refinement step: residual, one 16-bit V-cycle on the scaled residual, update
    const unsigned int* kmax_bits = (const unsigned int*)(flags + 2);
    if (face)
      launch_pdl(k_resid64<true>, dim3(nb), dim3(kBlock), 0, stream, d0, ks, op, x64, b, r, partials, sc, kmax_bits, cfg.max_iter, 0);
    else
      launch_pdl(k_resid64<false>, dim3(nb), dim3(kBlock), 0, stream, d0, ks, op, x64, b, r, partials, sc, kmax_bits, cfg.max_iter, 0);
    vcycle(0);
    if (cfg.precision == OTM_PRECISION_MIXED_BF16)
      launch_pdl(k_update64<__nv_bfloat16>, dim3(ceil_div(nv, kBlock)), dim3(kBlock), 0, stream, nv, x64, (const __nv_bfloat16*)zv, sc);
    else
      launch_pdl(k_update64<__half>, dim3(ceil_div(nv, kBlock)), dim3(kBlock), 0, stream, nv, x64, (const __half*)zv, sc);
    launched(2);
  } else if (cfg.solver == OTM_SOLVER_PCG) {
    vcycle(0);
    pcg_direction((const float*)z, r, face, nb);
    launch_pdl(k_update_xr, dim3(nb), dim3(kBlock), 0, stream, nv, x, r, p, q, partials, sc, cfg.max_iter);
    launched(3);
  } else {
    if (face)
      launch_pdl(k_resid_norm<true>, dim3(nb), dim3(kBlock), 0, stream, d0, ks, op, x, b, r, partials, sc, cfg.max_iter);
    else
      launch_pdl(k_resid_norm<false>, dim3(nb), dim3(kBlock), 0, stream, d0, ks, op, x, b, r, partials, sc, cfg.max_iter);
    vcycle(0);
    launch_pdl(k_axpy_x, dim3(ceil_div(3 * nv, kBlock)), dim3(kBlock), 0, stream, nv, x, z, sc);
    launched(2);
  }
}

otm_status Homo::run_chunk(int iters) {
  OTM_TRY(join_coarse());
  if (!cfg.use_graphs) {
    for (int i = 0; i < iters; i++) iteration(i);
    OTM_CHECK_LAUNCH("iteration");
    return OTM_OK;
  }
  ChunkGraph* g = nullptr;
  for (auto& gg : graphs)
    if (gg.iters == iters && gg.solver == cfg.solver) g = &gg;
  if (!g) {
    graphs.push_back(ChunkGraph{});
    g = &graphs.back();
    g->iters = iters;
    g->solver = cfg.solver;
    cudaGraph_t graph;
    OTM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    for (int i = 0; i < iters; i++) iteration(i);
    capturing = false;
    cudaError_t e = cudaStreamEndCapture(stream, &graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    size_t nn = 0;
    cudaGraphGetNodes(graph, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    cudaGraphGetNodes(graph, nodes.data(), &nn);
    for (auto& nd : nodes) {
      cudaGraphNodeType t;
      if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) g->kernel_nodes++;
    }
    e = cudaGraphInstantiate(&g->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
  }
  OTM_CUDA(cudaGraphLaunch(g->exec, stream));
  count_launches(g->kernel_nodes);
  return OTM_OK;
}

// Right-hand sides, nullspace projection and initial residual of an FP32 solve from a zero
// initial guess (launches only; used by the serving form).
void Homo::launch_solve_init() {
  const Dims d0 = lv[0].d;
  const size_t nv = d0.nv();
  const int nb = reduce_blocks(nv);
  cudaMemsetAsync(x, 0, 3 * nv * sizeof(float), stream);
  k_rhs_mean<<<nb, kBlock, 0, stream>>>(d0, ks, ef, b, partials, means, &sc->counter[T_MEAN]);
  sc_host->tol = cfg.fem_rel_thres;
  cudaMemcpyAsync(&sc->tol, &sc_host->tol, sizeof(double), cudaMemcpyHostToDevice, stream);
  k_init_residual<false><<<nb, kBlock, 0, stream>>>(d0, ks, op, x, b, means, lv[0].f, partials, sc);
  launched(2);
}

// K^H of the current solutions (-> sc->kh), with the sensitivity of a pending
// heat_matrix_sensitivity call in the same element pass.
void Homo::launch_heat_matrix() {
  const Dims d0 = lv[0].d;
  const int nb = reduce_blocks(d0.nv());
  if (sens_req.on)
    k_elem_pass<true, true><<<nb, kBlock, 0, stream>>>(d0, ks, kraw, x, op, ef, sens_req.sw, cfg.power_penal,
                                                        sens_req.sens, sens_req.pitchT, partials, sc);
  else
    k_elem_pass<true, false><<<nb, kBlock, 0, stream>>>(d0, ks, kraw, x, op, ef, SensWeights{}, cfg.power_penal,
                                                         nullptr, 0, partials, sc);
  launched(1);
}

static SensWeights sens_weights(const float dC[9]) {
  SensWeights sw;
  int cnt = 0;
  for (int a = 0; a < 3; a++)
    for (int bq = a; bq < 3; bq++) sw.w[cnt++] = dC[a * 3 + bq] + (a != bq ? dC[bq * 3 + a] : 0.f);
  return sw;
}

// Solve the 3 load cases to the tolerance (MG_H::solveEquation, homogenization/MG.cpp:80-142;
// per-case warm start from the previous solution, homogenization/homogenization.cu:182-188).
// Import / coarsest status written by update() (pinned copy in flags_host).
otm_status Homo::check_flags() {
  if (flags_host[0]) {
    set_error("conductivity field holds a negative, NaN or Inf value");
    return OTM_ERR_NAN;
  }
  if (flags_host[1]) {
    set_error("coarsest-level matrix is not positive definite");
    return OTM_ERR_NAN;
  }
  return OTM_OK;
}

// The whole iteration loop as one graph: k_loop_start, then a conditional "while" node whose
// body is one iteration followed by k_loop_ctrl, so a solve needs no host round trip until it
// has finished. Built on first use (and again when the solver type changes).
otm_status Homo::launch_loop() {
  OTM_TRY(join_coarse());
  if (!loop_exec || loop_solver != cfg.solver) {
    if (loop_exec) cudaGraphExecDestroy(loop_exec);
    loop_exec = nullptr;
    cudaGraph_t g = nullptr;
    OTM_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h{};
    cudaGraphNode_t n0{}, n1{};
    cudaGraphNodeParams cp{};
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
      void* args0[] = {&sc, &h};
      cudaKernelNodeParams kp{};
      kp.func = (void*)k_loop_start;
      kp.gridDim = dim3(1);
      kp.blockDim = dim3(1);
      kp.sharedMemBytes = 0;
      kp.kernelParams = args0;
      kp.extra = nullptr;
      e = cudaGraphAddKernelNode(&n0, g, nullptr, 0, &kp);
    }
    if (e == cudaSuccess) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      e = cudaGraphAddNode(&n1, g, &n0, 1, &cp);
    }
    if (e == cudaSuccess) {
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        capturing = true;
        iteration(0);
        launch_pdl(k_loop_ctrl, dim3(1), dim3(1), 0, stream, sc, h, cfg.max_iter + 1);
        capturing = false;
        cudaGraph_t out = nullptr;
        e = cudaStreamEndCapture(stream, &out);
      }
      if (e == cudaSuccess) {
        size_t nn = 0;
        cudaGraphGetNodes(body, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        cudaGraphGetNodes(body, nodes.data(), &nn);
        loop_body_kernels = 0;
        for (auto& nd : nodes) {
          cudaGraphNodeType t;
          if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) loop_body_kernels++;
        }
      }
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&loop_exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      loop_exec = nullptr;
      return cuda_fail(e, "building the solve-loop graph");
    }
    loop_solver = cfg.solver;
  }
  OTM_CUDA(cudaGraphLaunch(loop_exec, stream));
  return OTM_OK;
}

// Right-hand sides, projection, initial residual (all solver forms).
void Homo::launch_solve_start() {
  const Dims d0 = lv[0].d;
  const size_t nv = d0.nv();
  const int nb = reduce_blocks(nv);
  // right-hand sides and their means; the initial residual kernel projects b off the constants
  k_rhs_mean<<<nb, kBlock, 0, stream>>>(d0, ks, ef, b, partials, means, &sc->counter[T_MEAN]);
  sc_host->tol = cfg.fem_rel_thres;
  cudaMemcpyAsync(&sc->tol, &sc_host->tol, sizeof(double), cudaMemcpyHostToDevice, stream);
  if (mixed) {
    k_sub_bmean<<<ceil_div(nv, kBlock), kBlock, 0, stream>>>(nv, b, means);
    const unsigned int* kmax_bits = (const unsigned int*)(flags + 2);
    if (face)
      k_resid64<true><<<nb, kBlock, 0, stream>>>(d0, ks, op, x64, b, lv[0].f, partials, sc, kmax_bits, cfg.max_iter,
                                                 1);
    else
      k_resid64<false><<<nb, kBlock, 0, stream>>>(d0, ks, op, x64, b, lv[0].f, partials, sc, kmax_bits,
                                                  cfg.max_iter, 1);
  } else if (face) {
    k_init_residual<true><<<nb, kBlock, 0, stream>>>(d0, ks, op, x, b, means, lv[0].f, partials, sc);
  } else {
    k_init_residual<false><<<nb, kBlock, 0, stream>>>(d0, ks, op, x, b, means, lv[0].f, partials, sc);
  }
  launched(mixed ? 3 : 2);
}

// One solve from the current x with the iteration loop on the device: start kernels, the loop
// graph, the FP32 copy of a mixed solution, optionally the K^H reduction, then the flags and
// solve scalars to pinned memory. Launches only; the caller waits on the stream and then reads
// flags_host / sc_host.
otm_status Homo::launch_device_solve(bool with_heat) {
  const size_t nv = lv[0].d.nv();
  launch_solve_start();  // needs only the conductivities: runs alongside the coarse chain
  OTM_CHECK_LAUNCH("solve init");
  const int L = int(lv.size());
  if (coarse_pending && L > 1 && cluster_l != 0 && tail_l != 0) {
    // the first iteration as direct launches: its fine-level pre-smoothing, residual and
    // restriction need no coarse operator and overlap the rest of the coarse chain
    join_in_cycle = true;
    iteration(0);
    join_in_cycle = false;
    OTM_CHECK_LAUNCH("first iteration");
  }
  OTM_TRY(join_coarse());
  OTM_TRY(launch_loop());
  if (mixed) {
    k_x64_to_x<<<ceil_div(3 * nv, kBlock), kBlock, 0, stream>>>(3 * nv, x64, x);
    launched(1);
  }
  if (with_heat) launch_heat_matrix();
  OTM_CHECK_LAUNCH("solve");
  OTM_CUDA(cudaMemcpyAsync(flags_host, flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream));
  OTM_CUDA(cudaMemcpyAsync(sc_host, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, stream));
  return OTM_OK;
}

// Solve the 3 load cases to the tolerance (MG_H::solveEquation, homogenization/MG.cpp:80-142;
// iterations PCG or stationary V-cycles). With graphs and without profiling the iteration loop
// runs on the device (launch_loop) and the host waits once; with with_heat the K^H reduction
// is queued before that wait (heat_ready tells the caller).
otm_status Homo::solve_impl(bool with_heat) {
  const Dims d0 = lv[0].d;
  const size_t nv = d0.nv();
  const bool device_loop = cfg.use_graphs && !cfg.profile;
  heat_ready = false;
  if (!device_loop) {
    OTM_TRY(join_coarse());
    OTM_CUDA(cudaMemcpyAsync(flags_host, flags, 2 * sizeof(int), cudaMemcpyDeviceToHost, stream));
    OTM_CUDA(cudaStreamSynchronize(stream));
    OTM_TRY(check_flags());
  }
  for (int attempt = 0; attempt < 2; attempt++) {
    if (!cfg.warm_start || attempt > 0) {
      OTM_CUDA(cudaMemsetAsync(x, 0, 3 * nv * sizeof(float), stream));
      if (mixed) OTM_CUDA(cudaMemsetAsync(x64, 0, 3 * nv * sizeof(double), stream));
    }
    if (device_loop) {
      OTM_TRY(launch_device_solve(with_heat));
      OTM_CUDA(cudaStreamSynchronize(stream));
      OTM_TRY(check_flags());
      count_launches(1 + loop_body_kernels * uint64_t(sc_host->loop));
      heat_ready = with_heat;
    } else {
      launch_solve_start();
      OTM_CHECK_LAUNCH("solve init");
      int nlaunched = 0, iter_before = 0;
      bool first_check = true;
      while (true) {
        OTM_CUDA(cudaMemcpyAsync(sc_host, sc, sizeof(SolveScalars), cudaMemcpyDeviceToHost, stream));
        OTM_CUDA(cudaStreamSynchronize(stream));
        if (cfg.profile && !first_check) {
          const int ran = sc_host->iter - iter_before;
          for (int j = 0; j < ran && j < kMaxChunk; j++) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, prof_ev[0][j], prof_ev[1][j]) == cudaSuccess) {
              prof_ms += ms;
              prof_sweeps++;
            } else {
              cudaGetLastError();  // a failed query must not surface at the next launch check
            }
          }
        }
        first_check = false;
        iter_before = sc_host->iter;
        if (sc_host->done || nlaunched >= cfg.max_iter) break;
        const int chunk = std::min(cfg.check_every, cfg.max_iter - nlaunched);
        OTM_TRY(run_chunk(chunk));
        nlaunched += chunk;
      }
    }
    stats.iterations = sc_host->iter;
    stats.refinements = mixed ? (cfg.solver == OTM_SOLVER_PCG ? sc_host->nrepl : sc_host->iter) : 0;
    for (int c = 0; c < 3; c++) stats.rel_res[c] = sc_host->relres[c];
    if (!sc_host->nan) break;
    // "numerical explode, resetting initial guess" (homogenization/MG.cpp:392-423): one
    // retry from a zero initial guess, then give up.
  }
  otm_status st = OTM_OK;
  if (sc_host->timeout) {
    set_error("a tile kernel's bounded wait for its right-hand-side copy ran out");
    st = OTM_ERR_TIMEOUT;
  } else if (sc_host->nan) {
    set_error("MG numerical explode");
    st = OTM_ERR_DIVERGED;
  } else {
    for (int c = 0; c < 3; c++)
      if (!(stats.rel_res[c] <= cfg.fem_rel_thres)) st = OTM_ERR_NOT_CONVERGED;
    if (st != OTM_OK) set_error("failed to converge within max_iter");
  }
  stats.status = st;
  solved = (st == OTM_OK || st == OTM_ERR_NOT_CONVERGED);
  if (mixed && !device_loop) {
    // FP32 copy of the FP64 solution for K^H, sensitivity and the solution accessors
    k_x64_to_x<<<ceil_div(3 * nv, kBlock), kBlock, 0, stream>>>(3 * nv, x64, x);
    launched(1);
  }
  return st;
}

// One V(pre, post) cycle on caller-given right-hand sides (MG_H::v_cycle, MG.cpp:46-71), with
// direct launches: the right-hand sides go into the fine level's f, the cycle runs from a zero
// correction with the handle's smoother, the correction is copied out. The cycle's kernels skip
// their work once a solve has set the done flag, so it is cleared first.
otm_status Homo::v_cycle_once(const float* f, float* u, int pre, int post) {
  if (mixed) {
    set_error("a single V-cycle is available in the FP32 form only");
    return OTM_ERR_UNSUPPORTED;
  }
  if (!updated) {
    set_error("update() must be called before a V-cycle");
    return OTM_ERR_STATE;
  }
  if (pre < 0 || post < 0 || pre + post == 0 || pre > 16 || post > 16) return invalid("need 1..16 smoothing sweeps");
  if (tiled && (pre == 0 || post == 0)) return invalid("the tiled smoother needs at least one sweep in each leg");
  const size_t nv = lv[0].d.nv();
  OTM_TRY(enter());
  OTM_TRY(join_coarse());
  OTM_CUDA(cudaMemcpyAsync(lv[0].f, f, 3 * nv * sizeof(float), cudaMemcpyDeviceToDevice, stream));
  OTM_CUDA(cudaMemsetAsync(&sc->done, 0, sizeof(int), stream));
  const int keep_pre = cfg.pre_smooth, keep_post = cfg.post_smooth;
  cfg.pre_smooth = pre;
  cfg.post_smooth = post;
  prof_slot = -1;
  vcycle(0);
  cfg.pre_smooth = keep_pre;
  cfg.post_smooth = keep_post;
  OTM_CHECK_LAUNCH("v_cycle");
  OTM_CUDA(cudaMemcpyAsync(u, fine_z(), 3 * nv * sizeof(float), cudaMemcpyDeviceToDevice, stream));
  return leave();
}

otm_status Homo::solve(otm_solve_stats* out) {
  if (!updated) {
    set_error("update() must be called before solving");
    return OTM_ERR_STATE;
  }
  OTM_TRY(enter());
  otm_status st = solve_impl();
  otm_status st2 = leave();
  if (out) *out = stats;
  return st != OTM_OK ? st : st2;
}

otm_status Homo::heat_matrix(double C[9], bool do_solve) {
  if (!C) return invalid("C is NULL");
  otm_status st = OTM_OK;
  if (do_solve && !updated) {
    set_error("update() must be called before solving");
    return OTM_ERR_STATE;
  }
  if (!do_solve && !solved) {
    set_error("no solution available");
    return OTM_ERR_STATE;
  }
  OTM_TRY(enter());
  heat_ready = false;
  if (do_solve) {
    st = solve_impl(true);
    if (st != OTM_OK && st != OTM_ERR_NOT_CONVERGED) {
      leave();
      return st;
    }
  }
  if (!heat_ready) {
    launch_heat_matrix();
    OTM_CHECK_LAUNCH("k_elem_pass");
    OTM_CUDA(cudaMemcpyAsync(sc_host->kh, sc->kh, 6 * sizeof(double), cudaMemcpyDeviceToHost, stream));
    OTM_CUDA(cudaStreamSynchronize(stream));
  }
  int cnt = 0;
  for (int a = 0; a < 3; a++)
    for (int bq = a; bq < 3; bq++) {
      C[a * 3 + bq] = sc_host->kh[cnt];
      C[bq * 3 + a] = sc_host->kh[cnt];
      cnt++;
    }
  OTM_TRY(leave());
  return st;
}

otm_status Homo::sensitivity(const float dC[9], float* sens, int pitchT, int lexi) {
  if (!dC || !sens) return invalid("NULL argument");
  if (!solved) {
    set_error("sensitivity needs a solved state (call heat_matrix first)");
    return OTM_ERR_STATE;
  }
  const Dims d0 = lv[0].d;
  if (!lexi || pitchT <= 0) pitchT = d0.nx;
  if (pitchT < d0.nx) return invalid("pitchT smaller than the x resolution");
  const SensWeights sw = sens_weights(dC);
  OTM_TRY(enter());
  const size_t nruns = size_t((d0.nx + kRun - 1) / kRun) * d0.ny * d0.nz;
  k_elem_pass<false, true><<<ceil_div(nruns, kBlock), kBlock, 0, stream>>>(d0, ks, kraw, x, op, ef, sw,
                                                                           cfg.power_penal, sens, pitchT, nullptr,
                                                                           nullptr);
  OTM_CHECK_LAUNCH("k_elem_pass");
  launched(1);
  return leave();
}

// heat_matrix and sensitivity(dC) in one element pass, for a dC known before K^H (a linear
// objective): the solve, then one kernel that emits both.
otm_status Homo::heat_matrix_sensitivity(double C[9], const float dC[9], float* sens, int pitchT, int lexi) {
  if (!C || !dC || !sens) return invalid("NULL argument");
  const Dims d0 = lv[0].d;
  if (!lexi || pitchT <= 0) pitchT = d0.nx;
  if (pitchT < d0.nx) return invalid("pitchT smaller than the x resolution");
  sens_req.on = true;
  sens_req.sw = sens_weights(dC);
  sens_req.sens = sens;
  sens_req.pitchT = pitchT;
  const otm_status st = heat_matrix(C, true);
  sens_req.on = false;
  return st;
}

otm_status Homo::element_energy(float* out) {
  if (!out) return invalid("NULL argument");
  if (!solved) {
    set_error("no solution available");
    return OTM_ERR_STATE;
  }
  OTM_TRY(enter());
  const Dims d0 = lv[0].d;
  k_energy_fields<<<ceil_div(d0.nv(), kBlock), kBlock, 0, stream>>>(d0, x, op, ef, out);
  OTM_CHECK_LAUNCH("k_energy_fields");
  launched(1);
  return leave();
}

}  // namespace otm

// =========================================================================================
// C ABI
// =========================================================================================
using otm::Homo;

struct otm_homo {
  Homo impl;
};

extern "C" {

const char* otm_status_string(otm_status s) {
  switch (s) {
    case OTM_OK: return "ok";
    case OTM_ERR_INVALID_ARGUMENT: return "invalid argument";
    case OTM_ERR_UNSUPPORTED: return "unsupported";
    case OTM_ERR_CUDA: return "CUDA error";
    case OTM_ERR_OUT_OF_MEMORY: return "out of device memory";
    case OTM_ERR_NOT_CONVERGED: return "not converged";
    case OTM_ERR_DIVERGED: return "diverged";
    case OTM_ERR_NAN: return "NaN or Inf";
    case OTM_ERR_BUDGET: return "over memory budget";
    case OTM_ERR_STATE: return "call out of order";
    case OTM_ERR_TIMEOUT: return "timeout";
    case OTM_ERR_CANCELLED: return "cancelled";
    case OTM_ERR_NOT_READY: return "not ready";
  }
  return "unknown status";
}

const char* otm_last_error(void) { return otm::g_last_error.c_str(); }

int otm_abi_version(void) { return OTM_ABI_VERSION; }

otm_status otm_config_init(otm_config* cfg) {
  if (!cfg) return OTM_ERR_INVALID_ARGUMENT;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->reso[0] = cfg->reso[1] = cfg->reso[2] = 128;  // cmdline.cpp:6-8
  cfg->fem_rel_thres = 0.01;                         // cmdline.cpp:28
  cfg->max_iter = 200;                               // MG.cpp:382
  cfg->pre_smooth = 1;
  cfg->post_smooth = 1;
  cfg->solver = OTM_SOLVER_PCG;
  cfg->precision = OTM_PRECISION_FP32;
  cfg->coarsest_max_dof = 64;
  cfg->power_penal = 1.0f;  // homogenization.h:22
  cfg->warm_start = 1;
  cfg->check_every = 4;
  cfg->use_graphs = 1;
  cfg->profile = 0;
  cfg->cluster_cycle = 1;
  cfg->smoother = OTM_SMOOTHER_TILED;
  return OTM_OK;
}

otm_status otm_homo_create(const otm_config* cfg, otm_homo** out) {
  if (!cfg || !out) return OTM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  otm_homo* h = new (std::nothrow) otm_homo();
  if (!h) return OTM_ERR_OUT_OF_MEMORY;
  otm_status st = h->impl.build(*cfg);
  if (st != OTM_OK) {
    delete h;
    return st;
  }
  *out = h;
  return OTM_OK;
}

otm_status otm_homo_destroy(otm_homo* h) {
  if (!h) return OTM_ERR_INVALID_ARGUMENT;
  cudaStreamSynchronize(h->impl.stream);
  delete h;
  return OTM_OK;
}

otm_status otm_homo_set_stream(otm_homo* h, void* stream) {
  if (!h) return OTM_ERR_INVALID_ARGUMENT;
  h->impl.user_stream = (cudaStream_t)stream;
  return OTM_OK;
}

otm_status otm_homo_get_config(const otm_homo* h, otm_config* cfg) {
  if (!h || !cfg) return OTM_ERR_INVALID_ARGUMENT;
  *cfg = h->impl.cfg;
  return OTM_OK;
}

otm_status otm_homo_set_tolerance(otm_homo* h, double tol) {
  if (!h || !(tol > 0.0)) return OTM_ERR_INVALID_ARGUMENT;
  h->impl.cfg.fem_rel_thres = tol;
  return OTM_OK;
}

otm_status otm_homo_update(otm_homo* h, const float* k_dev, int pitchT) {
  if (!h) return OTM_ERR_INVALID_ARGUMENT;
  return h->impl.update(k_dev, pitchT);
}

otm_status otm_homo_solve(otm_homo* h, otm_solve_stats* stats) {
  if (!h) return OTM_ERR_INVALID_ARGUMENT;
  return h->impl.solve(stats);
}

otm_status otm_homo_heat_matrix(otm_homo* h, double C[9]) {
  if (!h) return OTM_ERR_INVALID_ARGUMENT;
  return h->impl.heat_matrix(C, true);
}

otm_status otm_homo_heat_matrix_nosolve(otm_homo* h, double C[9]) {
  if (!h) return OTM_ERR_INVALID_ARGUMENT;
  return h->impl.heat_matrix(C, false);
}

otm_status otm_homo_sensitivity(otm_homo* h, const float dC[9], float* sens_dev, int pitchT, int lexi) {
  if (!h) return OTM_ERR_INVALID_ARGUMENT;
  return h->impl.sensitivity(dC, sens_dev, pitchT, lexi);
}

otm_status otm_homo_update_density(otm_homo* h, const int reso[3], const float* rho, int rho_pitchT, float* rho_f,
                                   float* dk, float* wsum, int weight_type, float radius, int periodic, float p,
                                   float k0, float kmin) {
  if (!h) return OTM_ERR_INVALID_ARGUMENT;
  const otm::Dims d = h->impl.lv[0].d;
  if (!reso || reso[0] != d.nx || reso[1] != d.ny || reso[2] != d.nz) {
    otm::set_error("reso differs from the handle's resolution");
    return OTM_ERR_INVALID_ARGUMENT;
  }
  otm::Homo::DensityArgs a{rho, rho_pitchT, rho_f, dk, wsum, weight_type, radius, periodic, p, k0, kmin};
  return h->impl.update_density(a);
}

otm_status otm_homo_heat_matrix_sensitivity(otm_homo* h, double C[9], const float dC[9], float* sens_dev, int pitchT,
                                            int lexi) {
  if (!h) return OTM_ERR_INVALID_ARGUMENT;
  return h->impl.heat_matrix_sensitivity(C, dC, sens_dev, pitchT, lexi);
}

otm_status otm_homo_element_energy(otm_homo* h, float* energy_dev) {
  if (!h) return OTM_ERR_INVALID_ARGUMENT;
  return h->impl.element_energy(energy_dev);
}

otm_status otm_homo_v_cycle(otm_homo* h, const float* f_dev, float* u_dev, int pre, int post) {
  if (!h || !f_dev || !u_dev) return OTM_ERR_INVALID_ARGUMENT;
  return h->impl.v_cycle_once(f_dev, u_dev, pre, post);
}

otm_status otm_homo_level(const otm_homo* h, int level, otm_level_info* info) {
  if (!h || !info) return OTM_ERR_INVALID_ARGUMENT;
  const Homo& H = h->impl;
  const int L = int(H.lv.size());
  if (level < 0 || level >= L) return OTM_ERR_INVALID_ARGUMENT;
  const otm::Level& lv = H.lv[level];
  info->levels = L;
  info->reso[0] = lv.d.nx;
  info->reso[1] = lv.d.ny;
  info->reso[2] = lv.d.nz;
  info->stencil = level > 0 || L == 1;
  const bool direct = level == L - 1 || (H.cluster_l >= 0 && level >= H.cluster_l) ||
                      (H.tail_l >= 0 && level >= H.tail_l);
  if (direct)
    info->smoother = -1;
  else if (level == 0)
    info->smoother = H.tiled ? OTM_SMOOTHER_TILED : OTM_SMOOTHER_COLOR;
  else
    info->smoother = lv.ctiled ? OTM_SMOOTHER_TILED : OTM_SMOOTHER_COLOR;
  return OTM_OK;
}

otm_status otm_homo_get_solution(otm_homo* h, int lcase, float* dst_dev) {
  if (!h || !dst_dev || lcase < 0 || lcase > 2) return OTM_ERR_INVALID_ARGUMENT;
  Homo& H = h->impl;
  const size_t nv = H.lv[0].d.nv();
  OTM_TRY(H.enter());
  OTM_CUDA(cudaMemcpyAsync(dst_dev, H.x + lcase * nv, nv * sizeof(float), cudaMemcpyDeviceToDevice, H.stream));
  return H.leave();
}

otm_status otm_homo_set_solution(otm_homo* h, int lcase, const float* src_dev) {
  if (!h || !src_dev || lcase < 0 || lcase > 2) return OTM_ERR_INVALID_ARGUMENT;
  Homo& H = h->impl;
  const size_t nv = H.lv[0].d.nv();
  OTM_TRY(H.enter());
  OTM_CUDA(cudaMemcpyAsync(H.x + lcase * nv, src_dev, nv * sizeof(float), cudaMemcpyDeviceToDevice, H.stream));
  if (H.mixed) {
    otm::k_x_to_x64<<<otm::ceil_div(nv, otm::kBlock), otm::kBlock, 0, H.stream>>>(nv, H.x + lcase * nv,
                                                                                 H.x64 + lcase * nv);
    H.launched(1);
  }
  return H.leave();
}

otm_status otm_homo_reset_displacement(otm_homo* h) {
  if (!h) return OTM_ERR_INVALID_ARGUMENT;
  Homo& H = h->impl;
  OTM_TRY(H.enter());
  OTM_CUDA(cudaMemsetAsync(H.x, 0, 3 * H.lv[0].d.nv() * sizeof(float), H.stream));
  if (H.mixed) OTM_CUDA(cudaMemsetAsync(H.x64, 0, 3 * H.lv[0].d.nv() * sizeof(double), H.stream));
  H.solved = false;
  return H.leave();
}

otm_status otm_homo_get_profile(otm_homo* h, otm_profile* prof, int reset) {
  if (!h || !prof) return OTM_ERR_INVALID_ARGUMENT;
  Homo& H = h->impl;
  const double nv = double(H.lv[0].d.nv());
  prof->sweeps = H.prof_sweeps;
  prof->sweep_ms = H.prof_ms;
  if (H.tiled) {
    // the post-smoothing leg, one launch per sweep: each reads u_in and k and writes u_out (storage
    // type, 3 cases) and reads f (FP32, 3 cases); the first also reads the coarse correction (FP32,
    // 3 cases, one eighth of the vertices)
    const double s = H.mixed ? 2.0 : 4.0;
    const int n = H.cfg.post_smooth;
    prof->sweep_bytes = nv * (n * (3.0 * s + s + 12.0 + 3.0 * s) + 12.0 / 8.0);
    prof->launches_per_sweep = n;
    prof->kernel_kind = 1;
  } else {
    prof->sweep_bytes = nv * (4.0 + 3.0 * (4.0 + 4.0 + 4.0));
    prof->launches_per_sweep = H.face ? 8 : 4;
    prof->kernel_kind = 0;
  }
  if (reset) {
    H.prof_sweeps = 0;
    H.prof_ms = 0.0;
  }
  return OTM_OK;
}

uint64_t otm_launch_count(void) { return otm::g_launches.load(); }

otm_status otm_homo_get_stats(const otm_homo* h, otm_solve_stats* stats) {
  if (!h || !stats) return OTM_ERR_INVALID_ARGUMENT;
  *stats = h->impl.stats;
  return OTM_OK;
}

}  // extern "C"
