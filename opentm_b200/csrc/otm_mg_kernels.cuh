// otm_mg_kernels.cuh -- sm_100a kernels of the periodic multigrid solver.
//
// Layout (all levels): vectors are lexicographic, x fastest, one periodic unknown per
// vertex, the 3 load cases stored case-major (case c at offset c * nv). The fine level is
// matrix-free from the element conductivity k_e (homogenization/grid.cu:318-471); coarse
// levels hold 27-point Galerkin stencils (homogenization/grid_ex.cu:16-227) in the
// "colour-blocked" order: stencil entry o of vertex (x,y,z) sits at
// st[o * nv + colour * nv/8 + sub], colour = x%2 + 2(y%2) + 4(z%2), sub the lexicographic
// index of (x/2, y/2, z/2), so that one Gauss-Seidel colour pass streams its coefficients.
// Stencil offset o = (ox+1) + 3(oy+1) + 9(oz+1).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "otm_common.cuh"

namespace otm {

// Entries of the trilinear element Laplacian by Hamming distance between local nodes:
// KE[i][j] = c[popc(i ^ j)] (templateMatrix.cpp:21-87 gives exactly this structure).
struct FineOp {
  float c0, c1, c2, c3;
};

// Scalars of an iterative solve kept on the device so no host round trip is needed per
// iteration.
struct SolveScalars {
  double bb[3];      // ||b||^2 per case
  double rz[3];      // r . z (projected) of the current iteration
  double alpha[3];
  double beta[3];
  double zmean[3];
  double rr[3];      // ||r||^2
  double relres[3];  // ||r|| / (||b|| + 1e-10)
  double tol;
  double kh[6];      // K^H unique entries 00 01 02 11 12 22
  double mean[3];    // scratch means
  int done;          // 1 once every case meets tol
  int iter;          // iterations performed
  int nan;           // 1 if a NaN/Inf appeared
  int first;         // 1 before the first beta
  unsigned int counter[8];  // last-block tickets
  // mixed precision: f is read as alpha_c * f by the inner cycle, x64 += xscale_c * u
  double fscale[3];
  double xscale[3];
  int loop;  // bodies run by the device-side solve loop of the current solve
  // mixed-precision PCG: exact FP64 residual replacements
  double rr_repl[3];  // ||r||^2 at the last replacement
  int repl;           // 1: the next replacement kernel recomputes r = b - A x64
  int nrepl;          // replacements (FP64 residuals) of the current solve
  int timeout;        // 1 if a kernel's bounded wait for its own asynchronous copy ran out
};

// Dynamic shared memory limit every large-shared-memory kernel is opted in to. It is one fixed
// value (the attribute is per function, not per launch), so handles of different sizes never
// lower each other's limit; every plan that uses dynamic shared memory stays below it.
constexpr int kMaxDynSmem = 200 * 1024;

enum Ticket { T_RZ = 0, T_PQ = 1, T_RR = 2, T_KH = 3, T_MEAN = 4, T_INIT = 5, T_RES = 6 };

__device__ __forceinline__ bool solve_done(const SolveScalars* sc) {
  return *((volatile const int*)&sc->done) != 0;
}

// Last-block ticket: returns true in every thread of the block that arrives last. The
// partial sums written before are visible to it (threadfence before the ticket).
__device__ __forceinline__ bool last_block(unsigned int* counter) {
  __shared__ bool is_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int prev = atomicAdd(counter, 1u);
    is_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (is_last) __threadfence();
  return is_last;
}

// As last_block for a block range of nblk blocks (batched launches: one range per request).
__device__ __forceinline__ bool last_block_n(unsigned int* counter, unsigned int nblk) {
  __shared__ bool is_last_n;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int prev = atomicAdd(counter, 1u);
    is_last_n = (prev == nblk - 1);
  }
  __syncthreads();
  if (is_last_n) __threadfence();
  return is_last_n;
}

// Fixed-order sum of NV partial columns (partials[b * NV + i], b < nb) inside one block.
// The partials of the other blocks are read from L2 (ld.global.cg: never a stale L1 line),
// with the loop unrolled so that several rounds of loads are in flight at once.
template <int NV>
__device__ __forceinline__ void reduce_partials(const double* partials, int nb, double (&out)[NV], double* smem) {
  double v[NV];
#pragma unroll
  for (int i = 0; i < NV; i++) v[i] = 0.0;
#pragma unroll 4
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
#pragma unroll
    for (int i = 0; i < NV; i++) v[i] += __ldcg(partials + b * NV + i);
  }
  block_reduce_f64<NV>(v, smem);
#pragma unroll
  for (int i = 0; i < NV; i++) out[i] = v[i];  // valid in thread 0
}

// ------------------------------------------------------------------------------------
// Fine level: operator coefficients from the 8 element conductivities around a vertex.
// k8[b] is the element whose lower corner is v - 1 + bits(b); it holds v as local node
// 7 - b (homogenization/homoCommon.cuh:287-355). A(v, v+o) = c[|o|_0] * (sum of k8[b] over
// the elements that contain both v and v+o): per axis o>0 needs bit 1, o<0 bit 0, o=0 any.
// ------------------------------------------------------------------------------------
template <int OX, int OY, int OZ>
__device__ __forceinline__ float ksum(const float (&k8)[8]) {
  float s = 0.f;
#pragma unroll
  for (int b = 0; b < 8; b++) {
    const int bx = b & 1, by = (b >> 1) & 1, bz = b >> 2;
    const bool okx = OX > 0 ? bx == 1 : (OX < 0 ? bx == 0 : true);
    const bool oky = OY > 0 ? by == 1 : (OY < 0 ? by == 0 : true);
    const bool okz = OZ > 0 ? bz == 1 : (OZ < 0 ? bz == 0 : true);
    if (okx && oky && okz) s += k8[b];
  }
  return s;
}

template <int O>
__device__ __forceinline__ float fine_coef(const float (&k8)[8], const FineOp& op) {
  constexpr int ox = O % 3 - 1, oy = (O / 3) % 3 - 1, oz = O / 9 - 1;
  constexpr int nzc = (ox != 0) + (oy != 0) + (oz != 0);
  const float c = nzc == 0 ? op.c0 : (nzc == 1 ? op.c1 : (nzc == 2 ? op.c2 : op.c3));
  return c * ksum<ox, oy, oz>(k8);
}

// Storage conversions of the fine-level fields (FP32, BF16 or FP16 storage, FP32 arithmetic).
__device__ __forceinline__ float ld(const float* p) { return *p; }
__device__ __forceinline__ float ld(const __nv_bfloat16* p) { return __bfloat162float(*p); }
__device__ __forceinline__ float ld(const __half* p) { return __half2float(*p); }
__device__ __forceinline__ void st(float* p, float v) { *p = v; }
__device__ __forceinline__ void st(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }
__device__ __forceinline__ void st(__half* p, float v) { *p = __float2half_rn(v); }

// Neighbour indices of (x,y,z) on a periodic grid: idx[o] for the 27 offsets.
struct Nbr {
  int xs[3];
  size_t rows[9];  // (ys[b] + ny * zs[c]) * nx for b,c in 0..2, index b + 3c
  __device__ __forceinline__ void init(const Dims& d, int x, int y, int z) {
    xs[0] = wrapm(x - 1, d.nx);
    xs[1] = x;
    xs[2] = wrapm(x + 1, d.nx);
    int ys[3] = {wrapm(y - 1, d.ny), y, wrapm(y + 1, d.ny)};
    int zs[3] = {wrapm(z - 1, d.nz), z, wrapm(z + 1, d.nz)};
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int b = 0; b < 3; b++) rows[b + 3 * c] = (size_t(ys[b]) + size_t(d.ny) * zs[c]) * d.nx;
  }
  __device__ __forceinline__ size_t at(int o) const { return rows[o / 3] + xs[o % 3]; }
};

// The 8 element conductivities around vertex (x,y,z): element lower corners x-1..x etc.
template <typename KT>
__device__ __forceinline__ void load_k8(const KT* __restrict__ ks, const Nbr& nb, float (&k8)[8]) {
#pragma unroll
  for (int b = 0; b < 8; b++) {
    const int bx = b & 1, by = (b >> 1) & 1, bz = b >> 2;
    // element lower corner (x-1+bx, y-1+by, z-1+bz) = neighbour offset (bx-1, by-1, bz-1)
    k8[b] = ld(ks + nb.rows[by + 3 * bz] + nb.xs[bx]);
  }
}

template <int O>
struct FineTerm {
  // whether offset O carries a coefficient when face entries (c1) are structurally zero
  static constexpr int ox = O % 3 - 1, oy = (O / 3) % 3 - 1, oz = O / 9 - 1;
  static constexpr int nzc = (ox != 0) + (oy != 0) + (oz != 0);
};

// acc[c] -= sum_{o != 0} A(v, v+o) u_c[v+o] over the 3 cases; returns the diagonal.
template <bool kFace, int NC, typename VT>
__device__ __forceinline__ float fine_offdiag(const float (&k8)[8], const FineOp& op, const Nbr& nb,
                                              const VT* u, size_t nv, float (&acc)[NC]) {
#pragma unroll
  for (int o = 0; o < 27; o++) {
    if (o == 13) continue;
    const int nzc = (o % 3 != 1) + ((o / 3) % 3 != 1) + (o / 9 != 1);
    if (!kFace && nzc == 1) continue;
    float coef;
    switch (o) {
#define OTM_FC(OO) \
  case OO:         \
    coef = fine_coef<OO>(k8, op); \
    break;
      OTM_FC(0) OTM_FC(1) OTM_FC(2) OTM_FC(3) OTM_FC(4) OTM_FC(5) OTM_FC(6) OTM_FC(7) OTM_FC(8)
      OTM_FC(9) OTM_FC(10) OTM_FC(11) OTM_FC(12) OTM_FC(14) OTM_FC(15) OTM_FC(16) OTM_FC(17)
      OTM_FC(18) OTM_FC(19) OTM_FC(20) OTM_FC(21) OTM_FC(22) OTM_FC(23) OTM_FC(24) OTM_FC(25) OTM_FC(26)
#undef OTM_FC
      default: coef = 0.f;
    }
    const size_t j = nb.at(o);
#pragma unroll
    for (int c = 0; c < NC; c++) acc[c] -= coef * ld(u + c * nv + j);
  }
  float ksum8 = 0.f;
#pragma unroll
  for (int b = 0; b < 8; b++) ksum8 += k8[b];
  return op.c0 * ksum8;
}

// One Gauss-Seidel colour pass on the fine level, omega = 1, all NC load cases
// (homogenization/grid.cu:318-471 without the periodic padding; the pinned Dirichlet vertex
// is replaced by mean projection in the outer solver).
// fscale (optional): per-case factor applied to f when it is read (scaled right-hand side of
// the mixed-precision inner cycle).
template <bool kFace, int NC, typename KT, typename VT>
__device__ __forceinline__ void gs_fine_body(const Dims& d, int color, const KT* __restrict__ ks, const FineOp& op,
                                             VT* u, const float* __restrict__ f, const double* fscale, size_t t) {
  const int hx = d.nx >> 1, hy = d.ny >> 1;
  const size_t nsub = d.nv() >> 3;
  if (t >= nsub) return;
  const Coord3 c3_ = split3(t, hx, hy);
    const int i = c3_.x, j = c3_.y, kq = c3_.z;
  const int x = 2 * i + (color & 1), y = 2 * j + ((color >> 1) & 1), z = 2 * kq + (color >> 2);
  Nbr nb;
  nb.init(d, x, y, z);
  float k8[8];
  load_k8(ks, nb, k8);
  const size_t nv = d.nv();
  const size_t v = nb.at(13);
  float acc[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) acc[c] = __ldg(f + c * nv + v) * (fscale ? float(fscale[c]) : 1.f);
  const float diag = fine_offdiag<kFace, NC>(k8, op, nb, u, nv, acc);
  const float inv = 1.0f / diag;
#pragma unroll
  for (int c = 0; c < NC; c++) st(u + c * nv + v, acc[c] * inv);
}

template <bool kFace, int NC, typename KT = float, typename VT = float>
__global__ void __launch_bounds__(kBlock) k_gs_fine(Dims d, int color, const KT* __restrict__ ks, FineOp op,
                                                     VT* u, const float* __restrict__ f, const SolveScalars* sc,
                                                     const double* fscale = nullptr) {
  pdl_wait();
  if (sc && solve_done(sc)) return;
  gs_fine_body<kFace, NC, KT, VT>(d, color, ks, op, u, f, fscale, size_t(blockIdx.x) * blockDim.x + threadIdx.x);
}

// Colour-pair pass on the fine level. With c1 == 0 (the cube element has no coupling between
// vertices one edge apart) colours (cx,cy,0) and (cx,cy,1) are not coupled, so both are
// updated in one launch: exactly a Gauss-Seidel sweep in the colour order 0,4,1,5,2,6,3,7.
// Each thread updates the vertical vertex pair (x, y, 2k) and (x, y, 2k+1), whose
// neighbourhoods share two of their four planes.
template <int NC, typename KT, typename VT>
__device__ __forceinline__ void gs_fine_pair_body(const Dims& d, int pair, const KT* __restrict__ ks,
                                                  const FineOp& op, VT* u, const float* __restrict__ f,
                                                  const double* fscale, size_t t) {
  const int hx = d.nx >> 1, hy = d.ny >> 1;
  const size_t nsub = d.nv() >> 3;
  if (t >= nsub) return;
  const Coord3 c3_ = split3(t, hx, hy);
    const int i = c3_.x, j = c3_.y, kq = c3_.z;
  const int x = 2 * i + (pair & 1), y = 2 * j + ((pair >> 1) & 1), z = 2 * kq;
  const size_t nv = d.nv();
  const int xs[3] = {wrapm(x - 1, d.nx), x, wrapm(x + 1, d.nx)};
  const int ys[3] = {wrapm(y - 1, d.ny), y, wrapm(y + 1, d.ny)};
  int zs[4];
#pragma unroll
  for (int a = 0; a < 4; a++) zs[a] = wrapm(z - 1 + a, d.nz);  // planes z-1 .. z+2
  // conductivities of the element planes z-1, z, z+1 (lower corners), 4 per plane
  float kk[3][4];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) {
      const int bx = b & 1, by = b >> 1;
      kk[a][b] = ld(ks + (size_t(ys[by]) + size_t(d.ny) * zs[a]) * d.nx + xs[bx]);
    }
#pragma unroll
  for (int h = 0; h < 2; h++) {  // h = 0: vertex at plane z (element planes 0,1); h = 1: z+1 (planes 1,2)
    float k8[8];
#pragma unroll
    for (int b = 0; b < 8; b++) k8[b] = kk[h + (b >> 2)][b & 3];
    const size_t v = (size_t(ys[1]) + size_t(d.ny) * zs[1 + h]) * d.nx + x;
    float acc[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) acc[c] = __ldg(f + c * nv + v) * (fscale ? float(fscale[c]) : 1.f);
#pragma unroll
    for (int o = 0; o < 27; o++) {
      const int ox = o % 3, oy = (o / 3) % 3, oz = o / 9;
      const int nzc = (ox != 1) + (oy != 1) + (oz != 1);
      if (nzc < 2) continue;  // self and the zero edge-neighbour entries
      float coef;
      switch (o) {
#define OTM_FC(OO) \
  case OO:         \
    coef = fine_coef<OO>(k8, op); \
    break;
        OTM_FC(0) OTM_FC(2) OTM_FC(6) OTM_FC(8) OTM_FC(1) OTM_FC(3) OTM_FC(5) OTM_FC(7) OTM_FC(9) OTM_FC(11)
        OTM_FC(15) OTM_FC(17) OTM_FC(18) OTM_FC(20) OTM_FC(24) OTM_FC(26) OTM_FC(19) OTM_FC(21) OTM_FC(23) OTM_FC(25)
#undef OTM_FC
        default: coef = 0.f;
      }
      const size_t jn = (size_t(ys[oy]) + size_t(d.ny) * zs[oz + h]) * d.nx + xs[ox];
#pragma unroll
      for (int c = 0; c < NC; c++) acc[c] -= coef * ld(u + c * nv + jn);
    }
    float ksum8 = 0.f;
#pragma unroll
    for (int b = 0; b < 8; b++) ksum8 += k8[b];
    const float inv = 1.0f / (op.c0 * ksum8);
#pragma unroll
    for (int c = 0; c < NC; c++) st(u + c * nv + v, acc[c] * inv);
  }
}

template <int NC, typename KT = float, typename VT = float>
__global__ void __launch_bounds__(kBlock) k_gs_fine_pair(Dims d, int pair, const KT* __restrict__ ks, FineOp op,
                                                          VT* u, const float* __restrict__ f, const SolveScalars* sc,
                                                          const double* fscale = nullptr) {
  pdl_wait();
  if (sc && solve_done(sc)) return;
  gs_fine_pair_body<NC, KT, VT>(d, pair, ks, op, u, f, fscale, size_t(blockIdx.x) * blockDim.x + threadIdx.x);
}

// The first colour-pair pass of a sweep that starts from u = 0: the neighbour products vanish,
// so the pass writes u = f / a_vv at the vertices of colour pair 0 (the vertical pair
// (2i, 2j, 2k), (2i, 2j, 2k+1)) and zero at the other six vertices of the 2x2x2 block, in place of
// the zero fill and the pass. a_vv, its summation order and the scaling of f are those of
// gs_fine_pair_body, so the values equal the pass's (which subtracts products with zero).
template <int NC, typename KT, typename VT>
__global__ void __launch_bounds__(kBlock) k_gs_fine_pair_first(Dims d, const KT* __restrict__ ks, FineOp op, VT* u,
                                                                const float* __restrict__ f, const SolveScalars* sc,
                                                                const double* fscale = nullptr) {
  pdl_wait();
  if (sc && solve_done(sc)) return;
  const int hx = d.nx >> 1, hy = d.ny >> 1;
  const size_t nsub = d.nv() >> 3;
  const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= nsub) return;
  const Coord3 c3_ = split3(t, hx, hy);
  const int x = 2 * c3_.x, y = 2 * c3_.y, z = 2 * c3_.z;
  const size_t nv = d.nv();
  const int xs[2] = {wrapm(x - 1, d.nx), x};
  const int ys[2] = {wrapm(y - 1, d.ny), y};
  int zs[3];
#pragma unroll
  for (int a = 0; a < 3; a++) zs[a] = wrapm(z - 1 + a, d.nz);  // element planes z-1 .. z+1
  float kk[3][4];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 4; b++) kk[a][b] = ld(ks + (size_t(ys[b >> 1]) + size_t(d.ny) * zs[a]) * d.nx + xs[b & 1]);
  float fv[2][NC];
#pragma unroll
  for (int h = 0; h < 2; h++)
#pragma unroll
    for (int c = 0; c < NC; c++)
      fv[h][c] = __ldg(f + c * nv + (size_t(y) + size_t(d.ny) * (z + h)) * d.nx + x) * (fscale ? float(fscale[c]) : 1.f);
#pragma unroll
  for (int h = 0; h < 2; h++) {
    float ksum8 = 0.f;
#pragma unroll
    for (int b = 0; b < 8; b++) ksum8 += kk[h + (b >> 2)][b & 3];
    const float inv = 1.0f / (op.c0 * ksum8);
    const size_t v = (size_t(y) + size_t(d.ny) * (z + h)) * d.nx + x;
#pragma unroll
    for (int c = 0; c < NC; c++) {
      VT* uc = u + c * nv;
      st(uc + v, fv[h][c] * inv);
      st(uc + v + 1, 0.f);
      st(uc + v + d.nx, 0.f);
      st(uc + v + d.nx + 1, 0.f);
    }
  }
}

// r = f - A u on the fine level for every vertex.
template <bool kFace, int NC, typename KT, typename VT>
__device__ __forceinline__ void resid_fine_body(const Dims& d, const KT* __restrict__ ks, const FineOp& op,
                                                const VT* __restrict__ u, const float* __restrict__ f,
                                                VT* __restrict__ r, const double* fscale, size_t v) {
  const size_t nv = d.nv();
  if (v >= nv) return;
  const Coord3 c3_ = split3(v, d.nx, d.ny);
    const int x = c3_.x, y = c3_.y, z = c3_.z;
  Nbr nb;
  nb.init(d, x, y, z);
  float k8[8];
  load_k8(ks, nb, k8);
  float acc[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) acc[c] = __ldg(f + c * nv + v) * (fscale ? float(fscale[c]) : 1.f);
  const float diag = fine_offdiag<kFace, NC>(k8, op, nb, u, nv, acc);
#pragma unroll
  for (int c = 0; c < NC; c++) st(r + c * nv + v, acc[c] - diag * ld(u + c * nv + v));
}

template <bool kFace, int NC, typename KT = float, typename VT = float>
__global__ void __launch_bounds__(kBlock) k_resid_fine(Dims d, const KT* __restrict__ ks, FineOp op,
                                                        const VT* __restrict__ u, const float* __restrict__ f,
                                                        VT* __restrict__ r, const SolveScalars* sc,
                                                        const double* fscale = nullptr) {
  pdl_wait();
  if (sc && solve_done(sc)) return;
  resid_fine_body<kFace, NC, KT, VT>(d, ks, op, u, f, r, fscale, size_t(blockIdx.x) * blockDim.x + threadIdx.x);
}

// ------------------------------------------------------------------------------------
// Coarse levels (27-point stencils, colour-blocked).
// ------------------------------------------------------------------------------------
__device__ __forceinline__ size_t cb_index(const Dims& d, int x, int y, int z) {
  const int hx = d.nx >> 1, hy = d.ny >> 1;
  const int color = (x & 1) + 2 * (y & 1) + 4 * (z & 1);
  return size_t(color) * (d.nv() >> 3) + size_t(x >> 1) + size_t(hx) * (size_t(y >> 1) + size_t(hy) * (z >> 1));
}

template <int NC>
__device__ __forceinline__ void gs_coarse_body(const Dims& d, int color, const float* __restrict__ st, float* u,
                                               const float* __restrict__ f, size_t t) {
  const int hx = d.nx >> 1, hy = d.ny >> 1;
  const size_t nsub = d.nv() >> 3;
  if (t >= nsub) return;
  const Coord3 c3_ = split3(t, hx, hy);
    const int i = c3_.x, j = c3_.y, kq = c3_.z;
  const int x = 2 * i + (color & 1), y = 2 * j + ((color >> 1) & 1), z = 2 * kq + (color >> 2);
  Nbr nb;
  nb.init(d, x, y, z);
  const size_t nv = d.nv();
  const size_t v = nb.at(13);
  const size_t sbase = size_t(color) * nsub + t;
  float acc[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) acc[c] = __ldg(f + c * nv + v);
#pragma unroll
  for (int o = 0; o < 27; o++) {
    if (o == 13) continue;
    const float s = __ldg(st + size_t(o) * nv + sbase);
    const size_t jn = nb.at(o);
#pragma unroll
    for (int c = 0; c < NC; c++) acc[c] -= s * u[c * nv + jn];
  }
  const float inv = 1.0f / __ldg(st + size_t(13) * nv + sbase);
#pragma unroll
  for (int c = 0; c < NC; c++) u[c * nv + v] = acc[c] * inv;
}

template <int NC>
__global__ void __launch_bounds__(kBlock) k_gs_coarse(Dims d, int color, const float* __restrict__ st, float* u,
                                                       const float* __restrict__ f, const SolveScalars* sc) {
  pdl_wait();
  if (sc && solve_done(sc)) return;
  gs_coarse_body<NC>(d, color, st, u, f, size_t(blockIdx.x) * blockDim.x + threadIdx.x);
}

// The first colour pass of a coarse-level sweep that starts from u = 0: u = f / a_vv at colour 0,
// zero at the other seven vertices of the 2x2x2 block, in place of the zero fill and the pass
// (the same values as gs_coarse_body, which subtracts products with zero).
template <int NC>
__global__ void __launch_bounds__(kBlock) k_gs_coarse_first(Dims d, const float* __restrict__ st, float* u,
                                                             const float* __restrict__ f, const SolveScalars* sc) {
  pdl_wait();
  if (sc && solve_done(sc)) return;
  const int hx = d.nx >> 1, hy = d.ny >> 1;
  const size_t nv = d.nv(), nsub = nv >> 3;
  const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= nsub) return;
  const Coord3 q = split3(t, hx, hy);
  const int x = 2 * q.x, y = 2 * q.y, z = 2 * q.z;
  const float inv = 1.0f / __ldg(st + size_t(13) * nv + t);  // colour 0: stencil index t
#pragma unroll
  for (int c = 0; c < NC; c++) {
    float* uc = u + c * nv;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const size_t v = (size_t(y) + size_t(d.ny) * (z + h)) * d.nx + x;
      const float a = h == 0 ? __ldg(f + c * nv + v) * inv : 0.f;
      uc[v] = a;
      uc[v + 1] = 0.f;
      uc[v + d.nx] = 0.f;
      uc[v + d.nx + 1] = 0.f;
    }
  }
}

template <int NC>
__device__ __forceinline__ void resid_coarse_body(const Dims& d, const float* __restrict__ st,
                                                  const float* __restrict__ u, const float* __restrict__ f,
                                                  float* __restrict__ r, size_t v) {
  const size_t nv = d.nv();
  if (v >= nv) return;
  const Coord3 c3_ = split3(v, d.nx, d.ny);
    const int x = c3_.x, y = c3_.y, z = c3_.z;
  Nbr nb;
  nb.init(d, x, y, z);
  const size_t sb = cb_index(d, x, y, z);
  float acc[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) acc[c] = __ldg(f + c * nv + v);
#pragma unroll
  for (int o = 0; o < 27; o++) {
    const float s = __ldg(st + size_t(o) * nv + sb);
    const size_t jn = nb.at(o);
#pragma unroll
    for (int c = 0; c < NC; c++) acc[c] -= s * __ldg(u + c * nv + jn);
  }
#pragma unroll
  for (int c = 0; c < NC; c++) r[c * nv + v] = acc[c];
}

template <int NC>
__global__ void __launch_bounds__(kBlock) k_resid_coarse(Dims d, const float* __restrict__ st,
                                                          const float* __restrict__ u, const float* __restrict__ f,
                                                          float* __restrict__ r, const SolveScalars* sc) {
  pdl_wait();
  if (sc && solve_done(sc)) return;
  resid_coarse_body<NC>(d, st, u, f, r, size_t(blockIdx.x) * blockDim.x + threadIdx.x);
}

// f_c(V) = sum_d w(d) r_f(2V + d), w = prod (1 - |d|/2): full weighting = P^T
// (homogenization/grid.cu:811-878).
template <int NC, typename VT>
__device__ __forceinline__ void restrict_body(const Dims& df, const Dims& dc, const VT* __restrict__ r,
                                              float* __restrict__ fc, size_t V) {
  const size_t nvc = dc.nv(), nvf = df.nv();
  if (V >= nvc) return;
  const Coord3 c3_ = split3(V, dc.nx, dc.ny);
    const int X = c3_.x, Y = c3_.y, Z = c3_.z;
  Nbr nb;
  nb.init(df, 2 * X, 2 * Y, 2 * Z);
  float acc[NC];
#pragma unroll
  for (int c = 0; c < NC; c++) acc[c] = 0.f;
#pragma unroll
  for (int o = 0; o < 27; o++) {
    const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = o / 9 - 1;
    const float w = (ox ? 0.5f : 1.f) * (oy ? 0.5f : 1.f) * (oz ? 0.5f : 1.f);
    const size_t j = nb.at(o);
#pragma unroll
    for (int c = 0; c < NC; c++) acc[c] += w * ld(r + c * nvf + j);
  }
#pragma unroll
  for (int c = 0; c < NC; c++) fc[c * nvc + V] = acc[c];
}

// pf / pf_bytes: data of a later kernel to bring into L2 (the coarse level's stencils, which the
// fine level's work evicts between two V-cycles), or null.
template <int NC, typename VT = float>
__global__ void __launch_bounds__(kBlock) k_restrict(Dims df, Dims dc, const VT* __restrict__ r,
                                                      float* __restrict__ fc, const SolveScalars* sc,
                                                      const void* pf, size_t pf_bytes) {
  l2_prefetch_share(pf, pf_bytes);  // data not written by the preceding kernels
  pdl_wait();
  if (sc && solve_done(sc)) return;
  restrict_body<NC, VT>(df, dc, r, fc, size_t(blockIdx.x) * blockDim.x + threadIdx.x);
}

// u_f += P u_c, trilinear interpolation (homogenization/grid.cu:881-940).
template <int NC, typename VT>
__device__ __forceinline__ void prolong_body(const Dims& df, const Dims& dc, const float* __restrict__ uc, VT* uf,
                                             size_t v) {
  const size_t nvc = dc.nv(), nvf = df.nv();
  if (v >= nvf) return;
  const Coord3 c3_ = split3(v, df.nx, df.ny);
    const int x = c3_.x, y = c3_.y, z = c3_.z;
  const int X0 = x >> 1, Y0 = y >> 1, Z0 = z >> 1;
  const int X1 = (x & 1) ? wrapm(X0 + 1, dc.nx) : X0;
  const int Y1 = (y & 1) ? wrapm(Y0 + 1, dc.ny) : Y0;
  const int Z1 = (z & 1) ? wrapm(Z0 + 1, dc.nz) : Z0;
  const float wx1 = (x & 1) ? 0.5f : 0.f, wy1 = (y & 1) ? 0.5f : 0.f, wz1 = (z & 1) ? 0.5f : 0.f;
  const float wx0 = 1.f - wx1, wy0 = 1.f - wy1, wz0 = 1.f - wz1;
  const size_t r00 = (size_t(Y0) + size_t(dc.ny) * Z0) * dc.nx, r10 = (size_t(Y1) + size_t(dc.ny) * Z0) * dc.nx;
  const size_t r01 = (size_t(Y0) + size_t(dc.ny) * Z1) * dc.nx, r11 = (size_t(Y1) + size_t(dc.ny) * Z1) * dc.nx;
#pragma unroll
  for (int c = 0; c < NC; c++) {
    const float* u = uc + c * nvc;
    const float a = wz0 * (wy0 * (wx0 * __ldg(u + r00 + X0) + wx1 * __ldg(u + r00 + X1)) +
                           wy1 * (wx0 * __ldg(u + r10 + X0) + wx1 * __ldg(u + r10 + X1))) +
                    wz1 * (wy0 * (wx0 * __ldg(u + r01 + X0) + wx1 * __ldg(u + r01 + X1)) +
                           wy1 * (wx0 * __ldg(u + r11 + X0) + wx1 * __ldg(u + r11 + X1)));
    st(uf + c * nvf + v, ld(uf + c * nvf + v) + a);
  }
}

template <int NC, typename VT = float>
__global__ void __launch_bounds__(kBlock) k_prolong(Dims df, Dims dc, const float* __restrict__ uc, VT* uf,
                                                     const SolveScalars* sc) {
  pdl_wait();
  if (sc && solve_done(sc)) return;
  prolong_body<NC, VT>(df, dc, uc, uf, size_t(blockIdx.x) * blockDim.x + threadIdx.x);
}

// u_f += P u_c with one thread per coarse vertex: its 2x2x2 block of coarse values (per case)
// is loaded once and interpolated to the 8 fine vertices (2X + dx, 2Y + dy, 2Z + dz), each with
// the expression and weights of prolong_body (the same values; 24 coarse loads per 8 fine
// vertices instead of per vertex). Needs even fine dimensions (every level with a coarser one).
template <int NC, typename VT>
__global__ void __launch_bounds__(kBlock) k_prolong8(Dims df, Dims dc, const float* __restrict__ uc, VT* uf,
                                                      const SolveScalars* sc) {
  pdl_wait();
  if (sc && solve_done(sc)) return;
  const size_t nvc = dc.nv(), nvf = df.nv();
  const size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= nvc) return;
  const Coord3 q = split3(t, dc.nx, dc.ny);
  const int Xs[2] = {q.x, wrapm(q.x + 1, dc.nx)};
  const int Ys[2] = {q.y, wrapm(q.y + 1, dc.ny)};
  const int Zs[2] = {q.z, wrapm(q.z + 1, dc.nz)};
#pragma unroll
  for (int c = 0; c < NC; c++) {
    const float* u = uc + c * nvc;
    float b[2][2][2];  // [z][y][x] offsets 0 / +1 from (X, Y, Z)
#pragma unroll
    for (int zi = 0; zi < 2; zi++)
#pragma unroll
      for (int yi = 0; yi < 2; yi++)
#pragma unroll
        for (int xi = 0; xi < 2; xi++)
          b[zi][yi][xi] = __ldg(u + (size_t(Ys[yi]) + size_t(dc.ny) * Zs[zi]) * dc.nx + Xs[xi]);
#pragma unroll
    for (int dz = 0; dz < 2; dz++)
#pragma unroll
      for (int dy = 0; dy < 2; dy++)
#pragma unroll
        for (int dx = 0; dx < 2; dx++) {
          const float wx1 = dx ? 0.5f : 0.f, wy1 = dy ? 0.5f : 0.f, wz1 = dz ? 0.5f : 0.f;
          const float wx0 = 1.f - wx1, wy0 = 1.f - wy1, wz0 = 1.f - wz1;
          const float a = wz0 * (wy0 * (wx0 * b[0][0][0] + wx1 * b[0][0][dx]) +
                                 wy1 * (wx0 * b[0][dy][0] + wx1 * b[0][dy][dx])) +
                          wz1 * (wy0 * (wx0 * b[dz][0][0] + wx1 * b[dz][0][dx]) +
                                 wy1 * (wx0 * b[dz][dy][0] + wx1 * b[dz][dy][dx]));
          const size_t v = (size_t(2 * q.x + dx) + size_t(df.nx) * (size_t(2 * q.y + dy) +
                                                                     size_t(df.ny) * (2 * q.z + dz)));
          st(uf + c * nvf + v, ld(uf + c * nvf + v) + a);
        }
  }
}

// ------------------------------------------------------------------------------------
// Galerkin coarse operators (homogenization/grid_ex.cu:16-227, restrict_stencil_*).
// ------------------------------------------------------------------------------------

// Level 1 from the fine conductivity: A_1(V, V+O) = sum over the 4^3 fine elements around
// 2V of k_e T[e][O], where T[e][O] = sum_ij P(p_i, V) KE_ij P(p_j, V+O) depends only on the
// element's position relative to 2V (tabulated on the host, 64 x 27, scaled by the element
// size). Element e = (ex,ey,ez) in 0..3 has its lower corner at 2V - 2 + (ex,ey,ez).
// kmax_bits (optional): divide the stencil by c0 * kmax, the normalisation of the
// mixed-precision inner operator (c0 is passed in c0).
static __global__ void __launch_bounds__(kBlock) k_galerkin_fine(Dims df, Dims dc, const float* __restrict__ ks,
                                                           const float* __restrict__ table, float* __restrict__ st,
                                                           int cb_out, const unsigned int* kmax_bits = nullptr,
                                                           float c0 = 1.f) {
  __shared__ float T[64 * 27];
  for (int i = threadIdx.x; i < 64 * 27; i += blockDim.x) T[i] = table[i];
  __syncthreads();
  const size_t nvc = dc.nv();
  const size_t V = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (V >= nvc) return;
  const Coord3 c3_ = split3(V, dc.nx, dc.ny);
    const int X = c3_.x, Y = c3_.y, Z = c3_.z;
  int xs[4], ys[4], zs[4];
#pragma unroll
  for (int a = 0; a < 4; a++) {
    xs[a] = wrapm(2 * X - 2 + a, df.nx);
    ys[a] = wrapm(2 * Y - 2 + a, df.ny);
    zs[a] = wrapm(2 * Z - 2 + a, df.nz);
  }
  float acc[27];
#pragma unroll
  for (int o = 0; o < 27; o++) acc[o] = 0.f;
#pragma unroll 1
  for (int ez = 0; ez < 4; ez++)
#pragma unroll
    for (int ey = 0; ey < 4; ey++) {
      const size_t row = (size_t(ys[ey]) + size_t(df.ny) * zs[ez]) * df.nx;
#pragma unroll
      for (int ex = 0; ex < 4; ex++) {
        const float k = __ldg(ks + row + xs[ex]);
        const float* Te = T + (ex + 4 * ey + 16 * ez) * 27;
#pragma unroll
        for (int o = 0; o < 27; o++) acc[o] += k * Te[o];
      }
    }
  const size_t out = cb_out ? cb_index(dc, X, Y, Z) : V;
  const float sc = kmax_bits ? 1.f / (c0 * __uint_as_float(*kmax_bits)) : 1.f;
#pragma unroll
  for (int o = 0; o < 27; o++) st[size_t(o) * nvc + out] = acc[o] * sc;
}

// Per-axis coarse targets of a fine offset t = d + o in [-2, 2]: the coarse offsets O with
// |t - 2 O| <= 1 and their trilinear weights.
__device__ __forceinline__ int axis_targets(int t, int (&O)[2], float (&w)[2]) {
  switch (t) {
    case -2: O[0] = -1; w[0] = 1.f; return 1;
    case -1: O[0] = -1; w[0] = 0.5f; O[1] = 0; w[1] = 0.5f; return 2;
    case 0: O[0] = 0; w[0] = 1.f; return 1;
    case 1: O[0] = 0; w[0] = 0.5f; O[1] = 1; w[1] = 0.5f; return 2;
    default: O[0] = 1; w[0] = 1.f; return 1;
  }
}

// Deeper levels: A_c(V, V+O) = sum_{d,o} P(2V+d, V) A_f(2V+d, o) P(2V+d+o, V+O).
// NSPLIT warps share 32 coarse vertices (one per lane): warp w forms the products of the fine
// offsets d in [w * 27 / NSPLIT, (w + 1) * 27 / NSPLIT) with compile-time offsets, in the order
// of d, and the partials of the warps are then summed in warp order through shared memory. With
// NSPLIT = 1 a thread forms all 729 products of its vertex, a chain of loads that makes every
// level's launch latency-bound; NSPLIT = 27 gives each warp a code path of its own.
template <int NSPLIT>
struct GalerkinShape {
  static constexpr int kGroups = NSPLIT >= 8 ? 1 : 8 / NSPLIT;  // 32-vertex groups per block
  static constexpr int kThreads = NSPLIT * 32 * kGroups;
  static constexpr size_t kSmem = size_t(kGroups) * NSPLIT * 27 * 32 * sizeof(float);
};

template <int DD>
__device__ __forceinline__ void galerkin_dd(const Dims& df, int X, int Y, int Z, const float* __restrict__ stf,
                                            float (&acc)[27]) {
  constexpr int dx = DD % 3 - 1, dy = (DD / 3) % 3 - 1, dz = DD / 9 - 1;
  const float wv = (dx ? 0.5f : 1.f) * (dy ? 0.5f : 1.f) * (dz ? 0.5f : 1.f);
  const size_t nvf = df.nv();
  const int fx = wrapm(2 * X + dx, df.nx), fy = wrapm(2 * Y + dy, df.ny), fz = wrapm(2 * Z + dz, df.nz);
  const size_t sb = cb_index(df, fx, fy, fz);
  float sv[27];
#pragma unroll
  for (int o = 0; o < 27; o++) sv[o] = __ldg(stf + size_t(o) * nvf + sb);
#pragma unroll
  for (int o = 0; o < 27; o++) {
    const float s = wv * sv[o];
    const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = o / 9 - 1;
    int Ox[2], Oy[2], Oz[2];
    float wx[2], wy[2], wz[2];
    const int nx = axis_targets(dx + ox, Ox, wx);
    const int ny = axis_targets(dy + oy, Oy, wy);
    const int nz = axis_targets(dz + oz, Oz, wz);
#pragma unroll
    for (int iz = 0; iz < 2; iz++)
#pragma unroll
      for (int iy = 0; iy < 2; iy++)
#pragma unroll
        for (int ix = 0; ix < 2; ix++) {
          if (ix < nx && iy < ny && iz < nz) {
            const int O = (Ox[ix] + 1) + 3 * (Oy[iy] + 1) + 9 * (Oz[iz] + 1);
            acc[O] += s * wx[ix] * wy[iy] * wz[iz];
          }
        }
  }
}

template <int D0, int D1>
__device__ __forceinline__ void galerkin_range(const Dims& df, int X, int Y, int Z, const float* __restrict__ stf,
                                               float (&acc)[27]) {
  galerkin_dd<D0>(df, X, Y, Z, stf, acc);
  if constexpr (D0 + 1 < D1) galerkin_range<D0 + 1, D1>(df, X, Y, Z, stf, acc);
}

// warp-uniform dispatch of warp w's offset range
template <int NSPLIT, int W>
__device__ __forceinline__ void galerkin_warp(int w, const Dims& df, int X, int Y, int Z,
                                              const float* __restrict__ stf, float (&acc)[27]) {
  constexpr int G = 27 / NSPLIT;
  if (w == W)
    galerkin_range<W * G, (W + 1) * G>(df, X, Y, Z, stf, acc);
  else if constexpr (W + 1 < NSPLIT)
    galerkin_warp<NSPLIT, W + 1>(w, df, X, Y, Z, stf, acc);
}

template <int NSPLIT>
__global__ void __launch_bounds__(GalerkinShape<NSPLIT>::kThreads)
    k_galerkin_coarse(Dims df, Dims dc, const float* __restrict__ stf, float* __restrict__ stc, int cb_out) {
  static_assert(27 % NSPLIT == 0, "the fine offsets split evenly");
  extern __shared__ float gpart[];  // [group][w][O][lane]
  const int warp = int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
  const int group = warp / NSPLIT, w = warp - group * NSPLIT;
  const size_t nvc = dc.nv();
  const size_t V = (size_t(blockIdx.x) * GalerkinShape<NSPLIT>::kGroups + group) * 32 + lane;
  const bool ok = V < nvc;
  const Coord3 c3_ = split3(ok ? V : 0, dc.nx, dc.ny);
  const int X = c3_.x, Y = c3_.y, Z = c3_.z;
  float acc[27];
#pragma unroll
  for (int o = 0; o < 27; o++) acc[o] = 0.f;
  galerkin_warp<NSPLIT, 0>(w, df, X, Y, Z, stf, acc);
  float* gp = gpart + size_t(group) * NSPLIT * 27 * 32;
#pragma unroll
  for (int o = 0; o < 27; o++) gp[(w * 27 + o) * 32 + lane] = acc[o];
  __syncthreads();
  for (int O = w; O < 27; O += NSPLIT) {
    float a = 0.f;
#pragma unroll
    for (int q = 0; q < NSPLIT; q++) a += gp[(q * 27 + O) * 32 + lane];
    if (ok) stc[size_t(O) * nvc + (cb_out ? cb_index(dc, X, Y, Z) : V)] = a;
  }
}

}  // namespace otm
