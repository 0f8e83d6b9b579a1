// otm_homo_impl.h -- the homogenization handle (internal).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "otm_mg_kernels.cuh"
#include "otm_solver_kernels.cuh"
#include "otm_cluster.cuh"
#include "otm_tail.cuh"
#include "otm_tile.cuh"
#include "otm_ctile.cuh"
#include "otm_template.h"

namespace otm {

// One multigrid level: 3 load cases of u (correction / solution), f (right-hand side) and
// r (residual scratch), plus the 27-point stencil on coarse levels.
struct Level {
  Dims d{};
  float* u = nullptr;
  float* f = nullptr;
  float* r = nullptr;
  float* st = nullptr;
  // coarse level smoothed by the tile kernels: second buffer of the sweep ping-pong
  bool ctiled = false;
  float* u2 = nullptr;
};

struct ChunkGraph {
  int iters = 0;
  int solver = 0;
  uint64_t kernel_nodes = 0;
  cudaGraphExec_t exec = nullptr;
};

constexpr int kMaxChunk = 64;

// otm_filter.cu: the density chain's forward pass into a handle's conductivity buffers.
otm_status density_forward_import(const Dims& d, const float* rho, int rho_pitchT, float* rho_f, float* dk,
                                  float* wsum, int weight_type, float radius, int periodic, float p, float k0,
                                  float kmin, float* kraw, float* ks, float pp, int* bad, cudaStream_t s);

struct Homo {
  otm_config cfg{};
  cudaStream_t stream = nullptr;       // private stream (graph capture needs a non-legacy stream)
  cudaStream_t user_stream = nullptr;  // ordering with the caller
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // The coarse operators (Galerkin stencils of levels >= 1 and the coarsest inverse) are built
  // on a side stream, concurrently with the solve start, which needs only the conductivities;
  // ev_coarse marks their completion and join_coarse() orders the main stream after it.
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_coarse = nullptr;
  bool coarse_pending = false;
  std::vector<Level> lv;
  TemplateMatrices tm{};
  FineOp op{};
  ElemFields ef{};
  bool face = false;
  // mixed precision: FP64 solution, 16-bit fine-level storage, normalised inner operator
  bool mixed = false;
  double* x64 = nullptr;
  void* k16 = nullptr;
  void* u16 = nullptr;
  void* r16 = nullptr;
  void* u2 = nullptr;  // tiled smoother: second buffer of the sweep ping-pong (fine storage type)
  FineOp op0{};  // op / c0
  float* ks = nullptr;    // solver conductivity 1e-9 + k^p
  float* kraw = nullptr;  // conductivity as imported
  float* b = nullptr;     // right-hand sides
  float* x = nullptr;     // solutions chi (kept for warm starts)
  float* p = nullptr;
  float* q = nullptr;
  double* Ainv = nullptr;
  int cluster_l = -1;       // first level handled by the cluster kernel (-1: none)
  size_t cluster_smem = 0;  // its dynamic shared memory per CTA
  ClDesc cl_desc{};         // its level layout (pointers filled per launch)
  // fine level smoothed by the tile kernels (one launch per smoothing leg); the post-smoothing
  // leg writes the preconditioned residual to the residual buffer (lv[0].r, or r16)
  bool tiled = false;
  double* tile_partials = nullptr;  // 3 partial sums per fine tile (k_tile_apply_dot)
  std::vector<int> cl_tab_host;  // plane tables of the cluster plan (kept: the copy is asynchronous)
  int* cl_tab = nullptr;          // their device copy
  CUtensorMap fmap{};  // TMA map of the fine right-hand side (3 cases, FP32) for the tile kernels
  int tail_l = -1;          // first level handled by the single-CTA tail kernel (-1: none)
  size_t tail_smem = 0;     // its dynamic shared memory
  int nc = 0;
  float* table = nullptr;
  SolveScalars* sc = nullptr;
  SolveScalars* sc_host = nullptr;
  double* partials = nullptr;
  double* means = nullptr;
  int* flags = nullptr;  // [0] bad import value, [1] coarsest not SPD
  // server mode: work on the server's stream, allocate from its memory pool, never block
  bool external = false;
  cudaMemPool_t pool = nullptr;
  std::vector<void*> allocations;
  // the first iteration of a device-loop solve runs outside the loop graph and waits for the
  // side stream's coarse chain only before its first coarse level (set while it is launched)
  bool join_in_cycle = false;
  size_t bytes_allocated = 0;
  std::vector<ChunkGraph> graphs;
  // the whole iteration loop as one graph (conditional while node), used without profiling
  cudaGraphExec_t loop_exec = nullptr;
  int loop_solver = -1;
  uint64_t loop_body_kernels = 0;
  int* flags_host = nullptr;  // pinned copy of flags[0..1]
  bool heat_ready = false;    // K^H of the last solve_impl(true) is already in sc_host->kh
  bool capturing = false;
  // profiling: events around the first fine-level post-smoothing sweep of iteration j of a chunk
  cudaEvent_t prof_ev[2][kMaxChunk] = {};
  int prof_slot = -1;
  int prof_sweeps = 0;
  double prof_ms = 0.0;
  bool updated = false;
  bool solved = false;
  otm_solve_stats stats{};

  ~Homo();
  otm_status alloc(void** p, size_t bytes);
  otm_status build(const otm_config& c, cudaStream_t ext_stream = nullptr, cudaMemPool_t ext_pool = nullptr,
                   bool external_mode = false);
  void launch_solve_init();
  // arguments of otm_homo_update_density (the density chain's forward pass, otm_density_forward)
  struct DensityArgs {
    const float* rho;
    int rho_pitchT;
    float *rho_f, *dk, *wsum;
    int weight_type;
    float radius;
    int periodic;
    float p, k0, kmin;
  };
  otm_status update_density(const DensityArgs& a);
  otm_status update_operators();
  void launch_heat_matrix();
  // the sensitivity that launch_heat_matrix emits in the same element pass (heat_matrix_sensitivity)
  struct SensRequest {
    bool on = false;
    SensWeights sw{};
    float* sens = nullptr;
    int pitchT = 0;
  } sens_req;
  otm_status heat_matrix_sensitivity(double C[9], const float dC[9], float* sens, int pitchT, int lexi);
  otm_status tile_attributes();
  otm_status join_coarse();
  otm_status enter();
  otm_status leave();
  otm_status update(const float* kin, int pitchT);
  void gs(int l, int color);
  template <typename T>
  void fine_ops16(int what, int color);
  void vcycle(int l);
  void vcycle_coarse_tiled(int l);
  template <typename KT, typename VT>
  void vcycle_fine_tiled(const KT* k, VT* u, VT* r, const FineOp& fop, const double* fs);
  // the fine level's V-cycle result (the preconditioned residual / correction)
  void* fine_z() const { return tiled ? (mixed ? r16 : (void*)lv[0].r) : (mixed ? u16 : (void*)lv[0].u); }
  // the stencils of coarse level l for the L2 prefetch of the restriction into it: null while the
  // side stream may still be writing them, on the coarsest level and for an unaligned buffer
  const void* st_prefetch(int l) const {
    if (coarse_pending || l <= 0 || l >= int(lv.size()) - 1 || !lv[l].st ||
        (reinterpret_cast<uintptr_t>(lv[l].st) & 15))
      return nullptr;
    return lv[l].st;
  }
  size_t st_prefetch_bytes(int l) const { return st_prefetch(l) ? 27 * lv[l].d.nv() * sizeof(float) : 0; }
  template <typename VT>
  void pcg_direction(const VT* z, const float* r, bool face, int nb);
  void gs_first(int l);
  void iteration(int j);
  void launched(uint64_t n) {
    if (!capturing) count_launches(n);
  }
  otm_status run_chunk(int iters);
  otm_status launch_loop();
  otm_status check_flags();
  void launch_solve_start();
  otm_status launch_device_solve(bool with_heat);
  otm_status solve_impl(bool with_heat = false);
  otm_status solve(otm_solve_stats* out);
  otm_status heat_matrix(double C[9], bool do_solve);
  otm_status sensitivity(const float dC[9], float* sens, int pitchT, int lexi);
  otm_status element_energy(float* out);
  otm_status v_cycle_once(const float* f, float* u, int pre, int post);
};

}  // namespace otm
