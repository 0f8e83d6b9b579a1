// otm_solver_kernels.cuh -- import, right-hand sides, coarsest direct solve, Krylov vector
// updates with deterministic FP64 reductions, K^H and sensitivity kernels.
#pragma once

#include <type_traits>

#include "otm_mg_kernels.cuh"

namespace otm {

// Element macro field (disp, 8 x 3) and load matrix (feMu, 8 x 3) of the template matrix,
// passed by value (homogenization/templateMatrix.cpp:84-85).
struct ElemFields {
  float disp[8][3];
  float feMu[8][3];
};

// Grid-stride partition with a fixed block count so reductions are deterministic. At most 8
// blocks per SM of a 148-SM B200: each thread sums several vertices and the last block reduces
// 1184 partials (128^3 OC step p50 3.06 ms, against 3.10-3.18 ms with 592, 888, 1024, 1480 or 2048
// blocks).
constexpr int kReduceBlocks = 8 * 148;
static_assert(kReduceBlocks <= kMaxPartials, "the partial buffers hold kMaxPartials blocks");
__host__ __device__ inline int reduce_blocks(size_t n) {
  size_t b = (n + kBlock - 1) / kBlock;
  if (b > size_t(kReduceBlocks)) b = kReduceBlocks;
  if (b < 1) b = 1;
  return int(b);
}

// Largest solver conductivity (positive floats order like their bit patterns).
static __global__ void k_kmax(size_t nv, const float* __restrict__ ks, unsigned int* kmax_bits) {
  unsigned int m = 0;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nv; i += size_t(gridDim.x) * blockDim.x)
    m = max(m, __float_as_uint(fmaxf(ks[i], 0.f)));
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) m = max(m, __shfl_down_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) atomicMax(kmax_bits, m);
}

// 16-bit copy of the normalised conductivity k / kmax for the mixed-precision inner cycle.
template <typename T>
__global__ void k_to16(size_t nv, const float* __restrict__ ks, const unsigned int* kmax_bits, T* k16) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  st(k16 + i, ks[i] / __uint_as_float(*kmax_bits));
}

// k_solver = 1e-9 + k^p from a pitched lexicographic field, k_raw keeps the input
// (Grid_H::update + update_rho_kernel, homogenization/grid.cu:2465-2504, 2646-2662; the
// floor is applied where the reference evaluates rho_penal, grid.cu:405).
static __global__ void k_import(Dims d, const float* __restrict__ kin, int pitchT, float p, float* __restrict__ ks,
                         float* __restrict__ kraw, int* bad) {
  const size_t nv = d.nv();
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= nv) return;
  const unsigned yz32 = unsigned(e) / unsigned(d.nx);
  const int x = int(unsigned(e) - yz32 * unsigned(d.nx));
  const size_t yz = yz32;
  const float k = __ldg(kin + yz * size_t(pitchT) + x);
  if (!(k >= 0.f) || !isfinite(k)) atomicOr(bad, 1);
  kraw[e] = k;
  ks[e] = kRhoPenalMin + (p == 1.f ? k : powf(k, p));
}

// f_c(v) = sum_{elements e around v} k_e feMu[local(v)][c] for the 3 load cases
// (enforce_unit_macro_strain_kernel_H, homogenization/grid.cu:1282-1327).
static __global__ void __launch_bounds__(kBlock) k_rhs(Dims d, const float* __restrict__ ks, ElemFields ef,
                                                 float* __restrict__ b) {
  const size_t nv = d.nv();
  const size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const Coord3 c3_ = split3(v, d.nx, d.ny);
    const int x = c3_.x, y = c3_.y, z = c3_.z;
  Nbr nb;
  nb.init(d, x, y, z);
  float k8[8];
  load_k8(ks, nb, k8);
  float acc[3] = {0.f, 0.f, 0.f};
#pragma unroll
  for (int bb = 0; bb < 8; bb++)
#pragma unroll
    for (int c = 0; c < 3; c++) acc[c] += k8[bb] * ef.feMu[7 - bb][c];
#pragma unroll
  for (int c = 0; c < 3; c++) b[c * nv + v] = acc[c];
}

// ---------------------------------------------------------------------------------------
// Deterministic reductions (fixed grid, fixed order, last-block finalisation).
// ---------------------------------------------------------------------------------------

// Right-hand sides (as k_rhs) and their per-case means -> bmean[0..2] (grid-stride, fixed grid).
// The initial guess is not projected: K^H, the energies and the sensitivity do not change when
// a constant is added to a case's solution (the element matrix annihilates constants), and
// every Krylov update adds a mean-free direction.
static __global__ void __launch_bounds__(kBlock) k_rhs_mean(Dims d, const float* __restrict__ ks, ElemFields ef,
                                                            float* __restrict__ b, double* partials, double* bmean,
                                                            unsigned int* counter) {
  __shared__ double smem[32 * 3];
  const size_t nv = d.nv();
  double v[3] = {0, 0, 0};
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nv; i += size_t(gridDim.x) * blockDim.x) {
    const Coord3 c3_ = split3(i, d.nx, d.ny);
    const int x = c3_.x, y = c3_.y, z = c3_.z;
    Nbr nb;
    nb.init(d, x, y, z);
    float k8[8];
    load_k8(ks, nb, k8);
    float acc[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int bb = 0; bb < 8; bb++)
#pragma unroll
      for (int c = 0; c < 3; c++) acc[c] += k8[bb] * ef.feMu[7 - bb][c];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      b[c * nv + i] = acc[c];
      v[c] += acc[c];
    }
  }
  block_reduce_f64<3>(v, smem);
  if (threadIdx.x == 0)
#pragma unroll
    for (int i = 0; i < 3; i++) partials[blockIdx.x * 3 + i] = v[i];
  if (last_block(counter)) {
    double r[3];
    reduce_partials<3>(partials, gridDim.x, r, smem);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int i = 0; i < 3; i++) bmean[i] = r[i] / double(nv);
      *counter = 0;
    }
  }
}

// b -= mean b per case (the mixed-precision start, whose residual kernel reads b).
static __global__ void __launch_bounds__(kBlock) k_sub_bmean(size_t nv, float* b, const double* bmean) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= nv) return;
#pragma unroll
  for (int c = 0; c < 3; c++) b[c * nv + i] -= float(bmean[c]);
}

// b -= mean b (per case, in place), r = b - A x on the fine level, ||b||^2 and ||r||^2 -> sc
// (start of a Krylov solve).
template <bool kFace>
__global__ void __launch_bounds__(kBlock) k_init_residual(Dims d, const float* __restrict__ ks, FineOp op,
                                                          const float* __restrict__ x, float* b,
                                                          const double* __restrict__ bmean, float* __restrict__ r,
                                                          double* partials, SolveScalars* sc) {
  __shared__ double smem[32 * 6];
  const size_t nv = d.nv();
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nv; i += size_t(gridDim.x) * blockDim.x) {
    const Coord3 c3_ = split3(i, d.nx, d.ny);
    const int xx = c3_.x, yy = c3_.y, zz = c3_.z;
    Nbr nb;
    nb.init(d, xx, yy, zz);
    float k8[8];
    load_k8(ks, nb, k8);
    float acc[3], bp[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      bp[c] = b[c * nv + i] - float(bmean[c]);
      b[c * nv + i] = bp[c];
      acc[c] = bp[c];
    }
    const float diag = fine_offdiag<kFace, 3>(k8, op, nb, x, nv, acc);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float rc = acc[c] - diag * x[c * nv + i];
      r[c * nv + i] = rc;
      const double bc = bp[c];
      v[c] += bc * bc;
      v[3 + c] += double(rc) * rc;
    }
  }
  block_reduce_f64<6>(v, smem);
  if (threadIdx.x == 0)
#pragma unroll
    for (int i = 0; i < 6; i++) partials[blockIdx.x * 6 + i] = v[i];
  if (last_block(&sc->counter[T_INIT])) {
    double t[6];
    reduce_partials<6>(partials, gridDim.x, t, smem);
    if (threadIdx.x == 0) {
      bool all = true, bad = false;
      for (int c = 0; c < 3; c++) {
        sc->bb[c] = t[c];
        sc->rr[c] = t[3 + c];
        const double rel = sqrt(t[3 + c]) / (sqrt(t[c]) + 1e-10);
        sc->relres[c] = rel;
        if (!(rel <= sc->tol)) all = false;
        if (!isfinite(rel)) bad = true;
      }
      sc->done = all ? 1 : 0;
      sc->nan = bad ? 1 : 0;
      sc->timeout = 0;
      sc->iter = 0;
      sc->first = 1;
      sc->counter[T_INIT] = 0;
    }
  }
}

// rho = r . z, zbar = mean z, rbar-correction; beta = rho / rho_old (0 on the first step).
// A 16-bit z (the mixed-precision V-cycle's result on the scaled residual) is read as
// xscale_c * u, in solution units.
template <typename VT = float>
__device__ __forceinline__ void dot_rz_body(size_t nv, const float* __restrict__ r, const VT* __restrict__ z,
                                            double* partials, SolveScalars* sc, unsigned int blk, unsigned int nblk) {
  constexpr bool kScaled = !std::is_same<VT, float>::value;
  __shared__ double smem[32 * 9];
  double zs[3] = {1.0, 1.0, 1.0};
  if (kScaled)
#pragma unroll
    for (int c = 0; c < 3; c++) zs[c] = sc->xscale[c];
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (!kScaled && (nv & 3) == 0) {
    // FP32 z: four consecutive vertices per step with 16-byte loads (case planes are 16-byte aligned
    // when nv is a multiple of 4)
    const size_t n4 = nv >> 2;
    const float4* r4 = reinterpret_cast<const float4*>(r);
    const float4* z4 = reinterpret_cast<const float4*>(z);
    for (size_t i = size_t(blk) * blockDim.x + threadIdx.x; i < n4; i += size_t(nblk) * blockDim.x) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float4 a = r4[c * n4 + i], b = __ldg(z4 + c * n4 + i);
        const double ra[4] = {a.x, a.y, a.z, a.w}, zb[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
        for (int e = 0; e < 4; e++) {
          v[c] += ra[e] * zb[e];
          v[3 + c] += zb[e];
          v[6 + c] += ra[e];
        }
      }
    }
  } else {
    for (size_t i = size_t(blk) * blockDim.x + threadIdx.x; i < nv; i += size_t(nblk) * blockDim.x) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const double rc = r[c * nv + i];
        const double zc = kScaled ? zs[c] * double(ld(z + c * nv + i)) : double(ld(z + c * nv + i));
        v[c] += rc * zc;
        v[3 + c] += zc;
        v[6 + c] += rc;
      }
    }
  }
  block_reduce_f64<9>(v, smem);
  if (threadIdx.x == 0)
#pragma unroll
    for (int i = 0; i < 9; i++) partials[blk * 9 + i] = v[i];
  if (last_block_n(&sc->counter[T_RZ], nblk)) {
    double t[9];
    reduce_partials<9>(partials, nblk, t, smem);
    if (threadIdx.x == 0) {
      for (int c = 0; c < 3; c++) {
        const double zbar = t[3 + c] / double(nv);
        // (z - zbar) . r = z . r - zbar * sum r
        const double rz = t[c] - zbar * t[6 + c];
        sc->zmean[c] = zbar;
        sc->beta[c] = sc->first ? 0.0 : (sc->rz[c] != 0.0 ? rz / sc->rz[c] : 0.0);
        sc->rz[c] = rz;
      }
      sc->first = 0;
      sc->counter[T_RZ] = 0;
    }
  }
}

template <typename VT>
__global__ void __launch_bounds__(kBlock) k_dot_rz(size_t nv, const float* __restrict__ r, const VT* __restrict__ z,
                                                   double* partials, SolveScalars* sc) {
  pdl_wait();
  if (solve_done(sc)) return;
  dot_rz_body<VT>(nv, r, z, partials, sc, blockIdx.x, gridDim.x);
}

// p = (z - zbar) + beta p
__device__ __forceinline__ void update_p_body(size_t nv, const float* __restrict__ z, float* p,
                                              const SolveScalars* sc, size_t i) {
  if (i >= nv) return;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float zb = float(sc->zmean[c]), be = float(sc->beta[c]);
    p[c * nv + i] = (z[c * nv + i] - zb) + be * p[c * nv + i];
  }
}

static __global__ void __launch_bounds__(kBlock) k_update_p(size_t nv, const float* __restrict__ z, float* p,
                                                     const SolveScalars* sc) {
  pdl_wait();
  if (solve_done(sc)) return;
  update_p_body(nv, z, p, sc, size_t(blockIdx.x) * blockDim.x + threadIdx.x);
}

// q = A p on the fine level and alpha = rho / (p . q).
template <bool kFace>
__device__ __forceinline__ void apply_dot_body(const Dims& d, const float* __restrict__ ks, const FineOp& op,
                                               const float* __restrict__ p, float* __restrict__ q, double* partials,
                                               SolveScalars* sc, unsigned int blk, unsigned int nblk) {
  __shared__ double smem[32 * 3];
  const size_t nv = d.nv();
  double v[3] = {0, 0, 0};
  for (size_t i = size_t(blk) * blockDim.x + threadIdx.x; i < nv; i += size_t(nblk) * blockDim.x) {
    const Coord3 c3_ = split3(i, d.nx, d.ny);
    const int xx = c3_.x, yy = c3_.y, zz = c3_.z;
    Nbr nb;
    nb.init(d, xx, yy, zz);
    float k8[8];
    load_k8(ks, nb, k8);
    float acc[3] = {0.f, 0.f, 0.f};
    const float diag = fine_offdiag<kFace, 3>(k8, op, nb, p, nv, acc);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float pc = __ldg(p + c * nv + i);
      const float qc = diag * pc - acc[c];
      q[c * nv + i] = qc;
      v[c] += double(pc) * qc;
    }
  }
  block_reduce_f64<3>(v, smem);
  if (threadIdx.x == 0)
#pragma unroll
    for (int i = 0; i < 3; i++) partials[blk * 3 + i] = v[i];
  if (last_block_n(&sc->counter[T_PQ], nblk)) {
    double t[3];
    reduce_partials<3>(partials, nblk, t, smem);
    if (threadIdx.x == 0) {
      for (int c = 0; c < 3; c++) sc->alpha[c] = t[c] != 0.0 ? sc->rz[c] / t[c] : 0.0;
      sc->counter[T_PQ] = 0;
    }
  }
}

template <bool kFace>
__global__ void __launch_bounds__(kBlock) k_apply_dot(Dims d, const float* __restrict__ ks, FineOp op,
                                                      const float* __restrict__ p, float* __restrict__ q,
                                                      double* partials, SolveScalars* sc) {
  pdl_wait();
  if (solve_done(sc)) return;
  apply_dot_body<kFace>(d, ks, op, p, q, partials, sc, blockIdx.x, gridDim.x);
}

// The search-direction update and the operator product in one pass:
//   p = (z - zbar) + beta p,  q = A p = A z + beta q,  alpha = rho / (p . q).
// A annihilates constants (periodic Laplacian), so A p follows from A z and the previous q
// without a second gather. beta == 0 (first iteration) ignores the old p and q entirely.
// A 16-bit z is xscale_c * u: the gather runs on u and A z = xscale_c * (A u).
template <bool kFace, typename VT>
__global__ void __launch_bounds__(kBlock) k_update_p_apply_dot(Dims d, const float* __restrict__ ks, FineOp op,
                                                               const VT* __restrict__ z, float* __restrict__ p,
                                                               float* __restrict__ q, double* partials,
                                                               SolveScalars* sc) {
  constexpr bool kScaled = !std::is_same<VT, float>::value;
  pdl_wait();
  if (solve_done(sc)) return;
  __shared__ double smem[32 * 3];
  const size_t nv = d.nv();
  float be[3], zb[3], zs[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    be[c] = float(sc->beta[c]);
    zb[c] = float(sc->zmean[c]);
    zs[c] = kScaled ? float(sc->xscale[c]) : 1.f;
  }
  double v[3] = {0, 0, 0};
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nv; i += size_t(gridDim.x) * blockDim.x) {
    const Coord3 c3_ = split3(i, d.nx, d.ny);
    const int xx = c3_.x, yy = c3_.y, zz = c3_.z;
    Nbr nb;
    nb.init(d, xx, yy, zz);
    float k8[8];
    load_k8(ks, nb, k8);
    float acc[3] = {0.f, 0.f, 0.f};
    const float diag = fine_offdiag<kFace, 3>(k8, op, nb, z, nv, acc);
    float po[3], qo[3];  // all loads of the vertex before its stores
#pragma unroll
    for (int c = 0; c < 3; c++) {
      po[c] = be[c] != 0.f ? p[c * nv + i] : 0.f;
      qo[c] = be[c] != 0.f ? q[c * nv + i] : 0.f;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      float zc = ld(z + c * nv + i);
      float az = diag * zc - acc[c];
      if (kScaled) {
        zc *= zs[c];
        az *= zs[c];
      }
      float pc = zc - zb[c], qc = az;
      if (be[c] != 0.f) {
        pc += be[c] * po[c];
        qc += be[c] * qo[c];
      }
      p[c * nv + i] = pc;
      q[c * nv + i] = qc;
      v[c] += double(pc) * qc;
    }
  }
  block_reduce_f64<3>(v, smem);
  if (threadIdx.x == 0)
#pragma unroll
    for (int i = 0; i < 3; i++) partials[blockIdx.x * 3 + i] = v[i];
  if (last_block_n(&sc->counter[T_PQ], gridDim.x)) {
    double t[3];
    reduce_partials<3>(partials, gridDim.x, t, smem);
    if (threadIdx.x == 0) {
      for (int c = 0; c < 3; c++) sc->alpha[c] = t[c] != 0.0 ? sc->rz[c] / t[c] : 0.0;
      sc->counter[T_PQ] = 0;
    }
  }
}

// x += alpha p, r -= alpha q, ||r||^2 -> relative residual and the done flag.
__device__ __forceinline__ void update_xr_body(size_t nv, float* __restrict__ x, float* __restrict__ r,
                                               const float* __restrict__ p,
                                               const float* __restrict__ q, double* partials, SolveScalars* sc,
                                               int max_iter, unsigned int blk, unsigned int nblk) {
  __shared__ double smem[32 * 3];
  float al[3];
#pragma unroll
  for (int c = 0; c < 3; c++) al[c] = float(sc->alpha[c]);
  double v[3] = {0, 0, 0};
  if ((nv & 3) == 0) {
    // four consecutive vertices per step with 16-byte accesses
    const size_t n4 = nv >> 2;
    float4* x4 = reinterpret_cast<float4*>(x);
    float4* r4 = reinterpret_cast<float4*>(r);
    const float4* p4 = reinterpret_cast<const float4*>(p);
    const float4* q4 = reinterpret_cast<const float4*>(q);
    for (size_t i = size_t(blk) * blockDim.x + threadIdx.x; i < n4; i += size_t(nblk) * blockDim.x) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const size_t j = c * n4 + i;
        float4 xv = x4[j], rv = r4[j];
        const float4 pv = p4[j], qv = q4[j];
        xv.x += al[c] * pv.x;
        xv.y += al[c] * pv.y;
        xv.z += al[c] * pv.z;
        xv.w += al[c] * pv.w;
        rv.x -= al[c] * qv.x;
        rv.y -= al[c] * qv.y;
        rv.z -= al[c] * qv.z;
        rv.w -= al[c] * qv.w;
        x4[j] = xv;
        r4[j] = rv;
        v[c] += double(rv.x) * rv.x + double(rv.y) * rv.y + double(rv.z) * rv.z + double(rv.w) * rv.w;
      }
    }
  } else {
    for (size_t i = size_t(blk) * blockDim.x + threadIdx.x; i < nv; i += size_t(nblk) * blockDim.x) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        x[c * nv + i] += al[c] * p[c * nv + i];
        const float rc = r[c * nv + i] - al[c] * q[c * nv + i];
        r[c * nv + i] = rc;
        v[c] += double(rc) * rc;
      }
    }
  }
  block_reduce_f64<3>(v, smem);
  if (threadIdx.x == 0)
#pragma unroll
    for (int i = 0; i < 3; i++) partials[blk * 3 + i] = v[i];
  if (last_block_n(&sc->counter[T_RR], nblk)) {
    double t[3];
    reduce_partials<3>(partials, nblk, t, smem);
    if (threadIdx.x == 0) {
      bool all = true, bad = false;
      for (int c = 0; c < 3; c++) {
        sc->rr[c] = t[c];
        const double rel = sqrt(t[c]) / (sqrt(sc->bb[c]) + 1e-10);
        sc->relres[c] = rel;
        if (!(rel <= sc->tol)) all = false;
        if (!isfinite(rel) || rel > 1e10) bad = true;
      }
      sc->iter += 1;
      if (bad) sc->nan = 1;
      if (all || bad || sc->iter >= max_iter) sc->done = 1;
      sc->counter[T_RR] = 0;
    }
  }
}

static __global__ void __launch_bounds__(kBlock) k_update_xr(size_t nv, float* x, float* r, const float* __restrict__ p,
                                                      const float* __restrict__ q, double* partials,
                                                      SolveScalars* sc, int max_iter) {
  pdl_wait();
  if (solve_done(sc)) return;
  update_xr_body(nv, x, r, p, q, partials, sc, max_iter, blockIdx.x, gridDim.x);
}

// Stationary V-cycle iteration: r = b - A x with ||r||^2 -> relres/done (MG_H::solveEquation,
// homogenization/MG.cpp:80-142), then x += z after the cycle (k_axpy_x).
template <bool kFace>
__global__ void __launch_bounds__(kBlock) k_resid_norm(Dims d, const float* __restrict__ ks, FineOp op,
                                                       const float* __restrict__ x, const float* __restrict__ b,
                                                       float* __restrict__ r, double* partials, SolveScalars* sc,
                                                       int max_iter) {
  pdl_wait();
  if (solve_done(sc)) return;
  __shared__ double smem[32 * 3];
  const size_t nv = d.nv();
  double v[3] = {0, 0, 0};
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nv; i += size_t(gridDim.x) * blockDim.x) {
    const Coord3 c3_ = split3(i, d.nx, d.ny);
    const int xx = c3_.x, yy = c3_.y, zz = c3_.z;
    Nbr nb;
    nb.init(d, xx, yy, zz);
    float k8[8];
    load_k8(ks, nb, k8);
    float acc[3];
#pragma unroll
    for (int c = 0; c < 3; c++) acc[c] = b[c * nv + i];
    const float diag = fine_offdiag<kFace, 3>(k8, op, nb, x, nv, acc);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float rc = acc[c] - diag * x[c * nv + i];
      r[c * nv + i] = rc;
      v[c] += double(rc) * rc;
    }
  }
  block_reduce_f64<3>(v, smem);
  if (threadIdx.x == 0)
#pragma unroll
    for (int i = 0; i < 3; i++) partials[blockIdx.x * 3 + i] = v[i];
  if (last_block(&sc->counter[T_RES])) {
    double t[3];
    reduce_partials<3>(partials, gridDim.x, t, smem);
    if (threadIdx.x == 0) {
      bool all = true, bad = false;
      for (int c = 0; c < 3; c++) {
        sc->rr[c] = t[c];
        const double rel = sqrt(t[c]) / (sqrt(sc->bb[c]) + 1e-10);
        sc->relres[c] = rel;
        if (!(rel <= sc->tol)) all = false;
        if (!isfinite(rel) || rel > 10.0) bad = true;  // "numerical explode", MG.cpp:392
      }
      if (bad) sc->nan = 1;
      if (all || bad || sc->iter >= max_iter) sc->done = 1;
      sc->counter[T_RES] = 0;
    }
  }
}

static __global__ void __launch_bounds__(kBlock) k_axpy_x(size_t nv, float* x, const float* __restrict__ z,
                                                   SolveScalars* sc) {
  pdl_wait();
  if (solve_done(sc)) return;
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < 3 * nv) x[i] += z[i];
  if (i == 0) sc->iter += 1;
}


// 27-point stencil of the fine operator in lexicographic order (used when the fine level is
// also the coarsest and is solved directly).
static __global__ void __launch_bounds__(kBlock) k_fine_stencil(Dims d, const float* __restrict__ ks, FineOp op,
                                                         float* __restrict__ st) {
  const size_t nv = d.nv();
  const size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const Coord3 c3_ = split3(v, d.nx, d.ny);
    const int x = c3_.x, y = c3_.y, z = c3_.z;
  Nbr nb;
  nb.init(d, x, y, z);
  float k8[8];
  load_k8(ks, nb, k8);
#define OTM_ST(OO) st[size_t(OO) * nv + v] = fine_coef<OO>(k8, op);
  OTM_ST(0) OTM_ST(1) OTM_ST(2) OTM_ST(3) OTM_ST(4) OTM_ST(5) OTM_ST(6) OTM_ST(7) OTM_ST(8)
  OTM_ST(9) OTM_ST(10) OTM_ST(11) OTM_ST(12) OTM_ST(13) OTM_ST(14) OTM_ST(15) OTM_ST(16) OTM_ST(17)
  OTM_ST(18) OTM_ST(19) OTM_ST(20) OTM_ST(21) OTM_ST(22) OTM_ST(23) OTM_ST(24) OTM_ST(25) OTM_ST(26)
#undef OTM_ST
}


// ---------------------------------------------------------------------------------------
// Mixed precision: FP64 iterative refinement around a 16-bit-storage V-cycle.
// ---------------------------------------------------------------------------------------

// r = b - A x64 with FP64 accumulation from the FP32 conductivity, written as FP32 into f;
// reduces ||r||^2 and max|r| per case (and ||b||^2 when init != 0), then sets the relative
// residual, the done flag and the scales of the next inner cycle:
// fscale = 1 / max|r|, xscale = max|r| / (c0 kmax).
template <bool kFace>
__global__ void __launch_bounds__(kBlock) k_resid64(Dims d, const float* __restrict__ ks, FineOp op,
                                                    const double* __restrict__ x64, const float* __restrict__ b,
                                                    float* __restrict__ f, double* partials, SolveScalars* sc,
                                                    const unsigned int* kmax_bits, int max_iter, int init) {
  pdl_wait();
  // init: 1 start of a solve, 0 stationary refinement step, 2 residual replacement of the
  // mixed PCG (runs only when the previous update asked for it)
  if (init != 1 && solve_done(sc)) return;
  if (init == 2 && !*((volatile const int*)&sc->repl)) return;
  __shared__ double smem[32 * 6];
  const size_t nv = d.nv();
  double v[6] = {0, 0, 0, 0, 0, 0};
  double mx[3] = {0, 0, 0};
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nv; i += size_t(gridDim.x) * blockDim.x) {
    const Coord3 c3_ = split3(i, d.nx, d.ny);
    const int xx = c3_.x, yy = c3_.y, zz = c3_.z;
    Nbr nb;
    nb.init(d, xx, yy, zz);
    float k8[8];
    load_k8(ks, nb, k8);
    double acc[3];
#pragma unroll
    for (int c = 0; c < 3; c++) acc[c] = double(b[c * nv + i]);
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
      for (int c = 0; c < 3; c++) acc[c] -= double(coef) * x64[c * nv + j];
    }
    float ksum8 = 0.f;
#pragma unroll
    for (int q = 0; q < 8; q++) ksum8 += k8[q];
    const double diag = double(op.c0 * ksum8);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const double rc = acc[c] - diag * x64[c * nv + i];
      f[c * nv + i] = float(rc);
      v[3 + c] += rc * rc;
      mx[c] = fmax(mx[c], fabs(rc));
      if (init == 1) {
        const double bc = b[c * nv + i];
        v[c] += bc * bc;
      }
    }
  }
  block_reduce_f64<6>(v, smem);
  // block max of the 3 max-norms (warp shuffles, then shared memory)
  __shared__ double smx[32 * 3];
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) mx[c] = fmax(mx[c], __shfl_down_sync(0xffffffffu, mx[c], off));
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int c = 0; c < 3; c++) smx[(threadIdx.x >> 5) * 3 + c] = mx[c];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < int(blockDim.x + 31) / 32; w++)
      for (int c = 0; c < 3; c++) mx[c] = fmax(mx[c], smx[w * 3 + c]);
#pragma unroll
    for (int i = 0; i < 6; i++) partials[blockIdx.x * 9 + i] = v[i];
#pragma unroll
    for (int c = 0; c < 3; c++) partials[blockIdx.x * 9 + 6 + c] = mx[c];
  }
  if (last_block(&sc->counter[T_RES])) {
    // parallel fixed-order finalisation: 6 sums and 3 maxima over the blocks' partials
    double t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 4
    for (int bq = threadIdx.x; bq < int(gridDim.x); bq += blockDim.x)
#pragma unroll
      for (int i = 0; i < 9; i++) {
        const double val = __ldcg(partials + bq * 9 + i);
        t[i] = i < 6 ? t[i] + val : fmax(t[i], val);
      }
    double ts[6];
#pragma unroll
    for (int i = 0; i < 6; i++) ts[i] = t[i];
    block_reduce_f64<6>(ts, smem);  // result in thread 0
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) t[6 + c] = fmax(t[6 + c], __shfl_down_sync(0xffffffffu, t[6 + c], off));
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
#pragma unroll
      for (int c = 0; c < 3; c++) smx[(threadIdx.x >> 5) * 3 + c] = t[6 + c];
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < int(blockDim.x + 31) / 32; w++)
        for (int c = 0; c < 3; c++) t[6 + c] = fmax(t[6 + c], smx[w * 3 + c]);
#pragma unroll
      for (int i = 0; i < 6; i++) t[i] = ts[i];
      const double kmax = double(__uint_as_float(*kmax_bits));
      bool all = true, bad = false;
      if (init == 1) {
        sc->iter = 0;
        sc->nan = 0;
        sc->timeout = 0;
        sc->first = 1;
        sc->nrepl = 0;
      }
      for (int c = 0; c < 3; c++) {
        if (init == 1) sc->bb[c] = t[c];
        sc->rr_repl[c] = t[3 + c];
        sc->rr[c] = t[3 + c];
        const double rel = sqrt(t[3 + c]) / (sqrt(sc->bb[c]) + 1e-10);
        sc->relres[c] = rel;
        if (!(rel <= sc->tol)) all = false;
        if (!isfinite(rel) || rel > 1e10) bad = true;
        const double rmax = t[6 + c] > 0.0 ? t[6 + c] : 1.0;
        sc->fscale[c] = 1.0 / rmax;
        sc->xscale[c] = rmax / (double(op.c0) * kmax);
      }
      if (bad) sc->nan = 1;
      sc->done = (all || bad || sc->iter >= max_iter) ? 1 : 0;
      sc->repl = 0;
      sc->nrepl += 1;
      sc->counter[T_RES] = 0;
    }
  }
}

// Mixed PCG step: x64 += alpha p (FP64), r -= alpha q, ||r||^2 and max|r| -> relative residual,
// the 16-bit cycle's scales for the next residual, and the replacement request: the next
// k_resid64(init = 2) recomputes r = b - A x64 exactly once the recursive residual claims
// convergence (convergence is only declared on a replaced residual) or has fallen 1e6-fold since
// the last replacement. The recursive residual is FP32 (r -= alpha q with q = A p in FP32): its
// drift from b - A x64 stays near FP32 rounding of the largest residual since the last
// replacement, so a replacement every six orders of magnitude keeps it far below any tolerance.
static __global__ void __launch_bounds__(kBlock) k_update_x64r(size_t nv, double* __restrict__ x64,
                                                               float* __restrict__ r, const float* __restrict__ p,
                                                               const float* __restrict__ q, double* partials,
                                                               SolveScalars* sc, const unsigned int* kmax_bits,
                                                               float c0, int max_iter) {
  pdl_wait();
  if (solve_done(sc)) return;
  __shared__ double smem[32 * 3];
  __shared__ double smx[32 * 3];
  double al[3];
#pragma unroll
  for (int c = 0; c < 3; c++) al[c] = sc->alpha[c];
  double v[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
  if ((nv & 3) == 0) {
    // four consecutive vertices per step: 16-byte accesses to the FP32 vectors, two to x64
    const size_t n4 = nv >> 2;
    float4* r4 = reinterpret_cast<float4*>(r);
    const float4* p4 = reinterpret_cast<const float4*>(p);
    const float4* q4 = reinterpret_cast<const float4*>(q);
    double2* x2 = reinterpret_cast<double2*>(x64);
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n4; i += size_t(gridDim.x) * blockDim.x) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const size_t j = c * n4 + i;
        const float4 pv = p4[j], qv = q4[j];
        float4 rv = r4[j];
        double2 xa = x2[2 * j], xb = x2[2 * j + 1];
        xa.x += al[c] * double(pv.x);
        xa.y += al[c] * double(pv.y);
        xb.x += al[c] * double(pv.z);
        xb.y += al[c] * double(pv.w);
        x2[2 * j] = xa;
        x2[2 * j + 1] = xb;
        const float a = float(al[c]);
        rv.x -= a * qv.x;
        rv.y -= a * qv.y;
        rv.z -= a * qv.z;
        rv.w -= a * qv.w;
        r4[j] = rv;
        v[c] += double(rv.x) * rv.x + double(rv.y) * rv.y + double(rv.z) * rv.z + double(rv.w) * rv.w;
        mx[c] = fmax(mx[c], fmax(fmax(fabs(double(rv.x)), fabs(double(rv.y))), fmax(fabs(double(rv.z)), fabs(double(rv.w)))));
      }
    }
  } else {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < nv; i += size_t(gridDim.x) * blockDim.x) {
#pragma unroll
      for (int c = 0; c < 3; c++) {
        x64[c * nv + i] += al[c] * double(p[c * nv + i]);
        const float rc = r[c * nv + i] - float(al[c]) * q[c * nv + i];
        r[c * nv + i] = rc;
        v[c] += double(rc) * rc;
        mx[c] = fmax(mx[c], fabs(double(rc)));
      }
    }
  }
  block_reduce_f64<3>(v, smem);
#pragma unroll
  for (int c = 0; c < 3; c++)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) mx[c] = fmax(mx[c], __shfl_down_sync(0xffffffffu, mx[c], off));
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int c = 0; c < 3; c++) smx[(threadIdx.x >> 5) * 3 + c] = mx[c];
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < int(blockDim.x + 31) / 32; w++)
      for (int c = 0; c < 3; c++) mx[c] = fmax(mx[c], smx[w * 3 + c]);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      partials[blockIdx.x * 6 + c] = v[c];
      partials[blockIdx.x * 6 + 3 + c] = mx[c];
    }
  }
  if (last_block(&sc->counter[T_RR])) {
    double t[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll 4
    for (int bq = threadIdx.x; bq < int(gridDim.x); bq += blockDim.x)
#pragma unroll
      for (int i = 0; i < 6; i++) {
        const double val = __ldcg(partials + bq * 6 + i);
        t[i] = i < 3 ? t[i] + val : fmax(t[i], val);
      }
    double ts[3] = {t[0], t[1], t[2]};
    block_reduce_f64<3>(ts, smem);
#pragma unroll
    for (int c = 0; c < 3; c++)
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) t[3 + c] = fmax(t[3 + c], __shfl_down_sync(0xffffffffu, t[3 + c], off));
    __syncthreads();
    if ((threadIdx.x & 31) == 0)
#pragma unroll
      for (int c = 0; c < 3; c++) smx[(threadIdx.x >> 5) * 3 + c] = t[3 + c];
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < int(blockDim.x + 31) / 32; w++)
        for (int c = 0; c < 3; c++) t[3 + c] = fmax(t[3 + c], smx[w * 3 + c]);
      const double kmax = double(__uint_as_float(*kmax_bits));
      bool all = true, bad = false, drop = false;
      for (int c = 0; c < 3; c++) {
        sc->rr[c] = ts[c];
        const double rel = sqrt(ts[c]) / (sqrt(sc->bb[c]) + 1e-10);
        sc->relres[c] = rel;
        if (!(rel <= sc->tol)) all = false;
        if (!isfinite(rel) || rel > 1e10) bad = true;
        if (ts[c] <= 1e-12 * sc->rr_repl[c]) drop = true;  // the norm fell 1e6-fold
        const double rmax = t[3 + c] > 0.0 ? t[3 + c] : 1.0;
        sc->fscale[c] = 1.0 / rmax;
        sc->xscale[c] = rmax / (double(c0) * kmax);
      }
      sc->iter += 1;
      if (bad) sc->nan = 1;
      if (all || drop) sc->repl = 1;
      if (bad || sc->iter >= max_iter) sc->done = 1;
      sc->counter[T_RR] = 0;
    }
  }
}

// x64 += xscale_c * u (the inner cycle's correction, 16-bit storage); counts the step.
template <typename VT>
__global__ void __launch_bounds__(kBlock) k_update64(size_t nv, double* x64, const VT* __restrict__ u,
                                                     SolveScalars* sc) {
  pdl_wait();
  if (solve_done(sc)) return;
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < nv) {
#pragma unroll
    for (int c = 0; c < 3; c++) x64[c * nv + i] += sc->xscale[c] * double(ld(u + c * nv + i));
  }
  if (i == 0) sc->iter += 1;
}

static __global__ void k_x64_to_x(size_t n, const double* __restrict__ x64, float* x) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) x[i] = float(x64[i]);
}

static __global__ void k_x_to_x64(size_t n, const float* __restrict__ x, double* x64) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) x64[i] = double(x[i]);
}

// ---------------------------------------------------------------------------------------
// Device-side solve loop: a CUDA graph "while" node runs one iteration per body until the
// solve is done, diverged, or `cap` bodies have run (the cap bounds the loop even if no
// kernel ever sets done).
// ---------------------------------------------------------------------------------------
static __global__ void k_loop_start(SolveScalars* sc, cudaGraphConditionalHandle h) {
  sc->loop = 0;
  cudaGraphSetConditional(h, (sc->done || sc->nan) ? 0u : 1u);
}

static __global__ void k_loop_ctrl(SolveScalars* sc, cudaGraphConditionalHandle h, int cap) {
  pdl_wait();
  const int l = sc->loop + 1;
  sc->loop = l;
  cudaGraphSetConditional(h, (!sc->done && !sc->nan && l < cap) ? 1u : 0u);
}

// ---------------------------------------------------------------------------------------
// Coarsest level: dense FP64 inverse of A_c + (alpha/n) 1 1^T (SPD on the periodic
// nullspace), built once per update; each V-cycle applies it as a mat-vec. Replaces the
// host BiCGSTAB(ILUT) + nullspace projection of Grid_H::solveHostEquation
// (homogenization/grid.cpp:272-310).
// ---------------------------------------------------------------------------------------
// With use_smem the matrix is assembled and inverted in dynamic shared memory (n^2 doubles)
// and copied to Aout at the end; otherwise it is worked on in place in Aout.
constexpr int kGjRegs = 4;  // matrix elements per thread of the register-buffered elimination
static __global__ void __launch_bounds__(1024) k_coarsest_build(Dims d, const float* __restrict__ st, double* Aout, int* status,
                                        int use_smem) {
  extern __shared__ double smA[];
  const int n = int(d.nv());
  double* A = use_smem ? smA : Aout;
  for (size_t i = threadIdx.x; i < size_t(n) * n; i += blockDim.x) A[i] = 0.0;
  __syncthreads();
  __shared__ double dsum;
  if (threadIdx.x == 0) dsum = 0.0;
  __syncthreads();
  // row v assembled by one thread (handles periodic aliasing of small dims)
  for (int v = threadIdx.x; v < n; v += blockDim.x) {
    const int x = v % d.nx, y = (v / d.nx) % d.ny, z = v / (d.nx * d.ny);
    for (int o = 0; o < 27; o++) {
      const int jx = (x + o % 3 - 1 + d.nx) % d.nx, jy = (y + (o / 3) % 3 - 1 + d.ny) % d.ny,
                jz = (z + o / 9 - 1 + d.nz) % d.nz;
      const int j = jx + d.nx * (jy + d.ny * jz);
      A[size_t(v) * n + j] += double(st[size_t(o) * n + v]);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int v = 0; v < n; v++) s += A[size_t(v) * n + v];
    dsum = s;
  }
  __syncthreads();
  const double alpha = dsum / double(n) / double(n);
  for (size_t i = threadIdx.x; i < size_t(n) * n; i += blockDim.x) A[i] += alpha;
  __syncthreads();
  // in-place Gauss-Jordan inversion without pivoting (SPD)
  const int nn = n * n;  // n <= 1024
  if (nn <= kGjRegs * int(blockDim.x)) {
    // small systems: every element of step k is computed from the step's old values into
    // registers, then written back (two barriers per pivot instead of four)
    double nw[kGjRegs];
    int ei[kGjRegs], ej[kGjRegs];  // (row, column) of the thread's elements, fixed over the pivots
#pragma unroll
    for (int e = 0; e < kGjRegs; e++) {
      const int idx = int(threadIdx.x) + e * int(blockDim.x);
      ei[e] = idx / n;
      ej[e] = idx - ei[e] * n;
    }
    for (int k = 0; k < n; k++) {
      const double pv = A[k * n + k];
      if (threadIdx.x == 0 && !(pv > 0.0)) *status = 1;
      const double pinv = 1.0 / pv;
#pragma unroll
      for (int e = 0; e < kGjRegs; e++) {
        const int idx = int(threadIdx.x) + e * int(blockDim.x);
        if (idx < nn) {
          const int i = ei[e], j = ej[e];
          const double a = A[idx];
          if (i == k)
            nw[e] = j == k ? pinv : a * pinv;
          else if (j == k)
            nw[e] = a * -pinv;
          else
            nw[e] = a - A[i * n + k] * (A[k * n + j] * pinv);
        }
      }
      __syncthreads();
#pragma unroll
      for (int e = 0; e < kGjRegs; e++) {
        const int idx = int(threadIdx.x) + e * int(blockDim.x);
        if (idx < nn) A[idx] = nw[e];
      }
      __syncthreads();
    }
    if (use_smem)
      for (int i = threadIdx.x; i < nn; i += blockDim.x) Aout[i] = A[i];
    return;
  }
  __shared__ double piv_inv;
  for (int k = 0; k < n; k++) {
    if (threadIdx.x == 0) {
      const double pv = A[size_t(k) * n + k];
      if (!(pv > 0.0)) *status = 1;
      piv_inv = 1.0 / pv;
    }
    __syncthreads();
    const double pinv = piv_inv;
    for (int j = threadIdx.x; j < n; j += blockDim.x)
      if (j != k) A[size_t(k) * n + j] *= pinv;
    __syncthreads();
    for (size_t idx = threadIdx.x; idx < size_t(n) * n; idx += blockDim.x) {
      const int i = int(idx / n), j = int(idx % n);
      if (i != k && j != k) A[idx] -= A[size_t(i) * n + k] * A[size_t(k) * n + j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      if (i != k) A[size_t(i) * n + k] *= -pinv;
    __syncthreads();
    if (threadIdx.x == 0) A[size_t(k) * n + k] = pinv;
    __syncthreads();
  }
  if (use_smem)
    for (size_t i = threadIdx.x; i < size_t(n) * n; i += blockDim.x) Aout[i] = A[i];
}

// u = Ainv (f - mean f) for the 3 cases (one block).
static __global__ void k_coarsest_solve(int n, const double* __restrict__ Ainv, const float* __restrict__ f, float* u,
                                 const SolveScalars* sc) {
  pdl_wait();
  if (sc && solve_done(sc)) return;
  extern __shared__ double bsh[];  // 3 * n
  __shared__ double mean[3];
  for (int i = threadIdx.x; i < 3 * n; i += blockDim.x) bsh[i] = f[i];
  __syncthreads();
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += bsh[threadIdx.x * n + i];
    mean[threadIdx.x] = s / n;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int j = 0; j < n; j++) {
      const double m = Ainv[size_t(j) * n + i];  // symmetric: column read is coalesced
      a0 += m * (bsh[j] - mean[0]);
      a1 += m * (bsh[n + j] - mean[1]);
      a2 += m * (bsh[2 * n + j] - mean[2]);
    }
    u[i] = float(a0);
    u[n + i] = float(a1);
    u[2 * n + i] = float(a2);
  }
}

// ---------------------------------------------------------------------------------------
// K^H and sensitivity (homogenization/homogenization.cu:13-153, 255-412).
// ---------------------------------------------------------------------------------------

// E_ab = d_a^T KE d_b for the 6 unique pairs, d_c = disp[:,c] - chi_c at the 8 corners.
__device__ __forceinline__ void elem_energy(const Dims& d, size_t e, const float* __restrict__ chi, const FineOp& op,
                                            const ElemFields& ef, float (&E)[6]) {
  const size_t nv = d.nv();
  const Coord3 c3_ = split3(e, d.nx, d.ny);
    const int x = c3_.x, y = c3_.y, z = c3_.z;
  const int x1 = wrapm(x + 1, d.nx), y1 = wrapm(y + 1, d.ny), z1 = wrapm(z + 1, d.nz);
  const size_t r00 = (size_t(y) + size_t(d.ny) * z) * d.nx, r10 = (size_t(y1) + size_t(d.ny) * z) * d.nx;
  const size_t r01 = (size_t(y) + size_t(d.ny) * z1) * d.nx, r11 = (size_t(y1) + size_t(d.ny) * z1) * d.nx;
  const size_t idx[8] = {r00 + x, r00 + x1, r10 + x, r10 + x1, r01 + x, r01 + x1, r11 + x, r11 + x1};
  // KE_ij depends only on the Hamming distance |i ^ j| (c0, c1, c2, c3 for 0..3 differing bits), so
  // the 8-point Walsh-Hadamard transform W diagonalises it: KE = W diag(lam) W / 8 with lam_k =
  // l(popcount k), l(0) = c0 + 3c1 + 3c2 + c3, l(1) = c0 + c1 - c2 - c3, l(2) = c0 - c1 - c2 + c3,
  // l(3) = c0 - 3c1 + 3c2 - c3. Then E_ab = sum_k lam_k/8 w_a[k] w_b[k] with w = W (disp - chi).
  float w[3][8];
#pragma unroll
  for (int c = 0; c < 3; c++) {
#pragma unroll
    for (int j = 0; j < 8; j++) w[c][j] = ef.disp[j][c] - __ldg(chi + c * nv + idx[j]);
#pragma unroll
    for (int s = 1; s < 8; s <<= 1)
#pragma unroll
      for (int i = 0; i < 8; i++)
        if (!(i & s)) {
          const float a = w[c][i], b = w[c][i | s];
          w[c][i] = a + b;
          w[c][i | s] = a - b;
        }
  }
  const float l0 = 0.125f * (op.c0 + 3.f * op.c1 + 3.f * op.c2 + op.c3);
  const float l1 = 0.125f * (op.c0 + op.c1 - op.c2 - op.c3);
  const float l2 = 0.125f * (op.c0 - op.c1 - op.c2 + op.c3);
  const float l3 = 0.125f * (op.c0 - 3.f * op.c1 + 3.f * op.c2 - op.c3);
  int cnt = 0;
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int bq = a; bq < 3; bq++) {
      const float* u = w[a];
      const float* v = w[bq];
      const float s1 = u[1] * v[1] + u[2] * v[2] + u[4] * v[4];
      const float s2 = u[3] * v[3] + u[5] * v[5] + u[6] * v[6];
      E[cnt++] = l0 * (u[0] * v[0]) + l1 * s1 + l2 * s2 + l3 * (u[7] * v[7]);
    }
}

// K^H_ab = sum_e k_e E_ab(e) / vol with FP64 accumulation (vol = 1), -> sc->kh;
// sens_e = p k^(p-1) sum_{a<=b} E_ab (dC_ab + [a != b] dC_ba); pitched lexicographic output
// with zeroed pitch padding (Sensitivity_kernel_opt_2_H + init_array, homogenization.cu:415-479).
struct SensWeights {
  float w[6];
};

// The element pass of K^H and of the sensitivity, either or both at once (the sensitivity kernel
// fused with the K^H kernel: one pass computes the element energies once and emits the FP64 K^H
// partials and sens_e). One thread takes a run of kRun consecutive elements along x: the faces
// x0 .. x0 + kRun of the run are gathered once (4 corners x 3 cases) and transformed over (y, z)
// once, and each element combines two neighbouring faces with the x stage of the Walsh-Hadamard
// transform, so neighbouring elements share a face's loads and butterflies (about a third of
// the instructions of elem_energy per element). The transform is linear, so W (disp - chi) =
// W disp - W chi with W disp a per-thread constant. sens: written when kSens, pitched by pitchT
// with the padding zeroed.
constexpr int kRun = 8;

__device__ __forceinline__ void face_wht(const float* __restrict__ chi, size_t nv, size_t i00, size_t i10, size_t i01,
                                         size_t i11, float (&F)[3][4]) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float* q = chi + c * nv;
    const float a = __ldg(q + i00), b = __ldg(q + i10), cc = __ldg(q + i01), e = __ldg(q + i11);
    const float p0 = a + b, p1 = a - b, p2 = cc + e, p3 = cc - e;  // y stage
    F[c][0] = p0 + p2;                                                // z stage
    F[c][1] = p1 + p3;
    F[c][2] = p0 - p2;
    F[c][3] = p1 - p3;
  }
}

template <bool kKH, bool kSens>
__global__ void __launch_bounds__(kBlock) k_elem_pass(Dims d, const float* __restrict__ ks,
                                                     const float* __restrict__ kraw, const float* __restrict__ chi,
                                                     FineOp op, ElemFields ef, SensWeights sw, float p,
                                                     float* __restrict__ sens, int pitchT, double* partials,
                                                     SolveScalars* sc) {
  __shared__ double smem[32 * 6];
  const size_t nv = d.nv();
  const int nx = d.nx, ny = d.ny, nrow = (nx + kRun - 1) / kRun;
  const size_t nruns = size_t(nrow) * ny * d.nz;
  // W disp per case (same butterflies, index bits x, y, z = 1, 2, 4)
  float dw[3][8];
#pragma unroll
  for (int c = 0; c < 3; c++) {
#pragma unroll
    for (int j = 0; j < 8; j++) dw[c][j] = ef.disp[j][c];
#pragma unroll
    for (int st = 1; st < 8; st <<= 1)
#pragma unroll
      for (int i = 0; i < 8; i++)
        if (!(i & st)) {
          const float a = dw[c][i], b = dw[c][i | st];
          dw[c][i] = a + b;
          dw[c][i | st] = a - b;
        }
  }
  const float l0 = 0.125f * (op.c0 + 3.f * op.c1 + 3.f * op.c2 + op.c3);
  const float l1 = 0.125f * (op.c0 + op.c1 - op.c2 - op.c3);
  const float l2 = 0.125f * (op.c0 - op.c1 - op.c2 + op.c3);
  const float l3 = 0.125f * (op.c0 - 3.f * op.c1 + 3.f * op.c2 - op.c3);
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (size_t r = size_t(blockIdx.x) * blockDim.x + threadIdx.x; r < nruns; r += size_t(gridDim.x) * blockDim.x) {
    const unsigned yz = unsigned(r / unsigned(nrow));
    const int x0 = int(r - size_t(yz) * nrow) * kRun;
    const int y = int(yz % unsigned(ny)), z = int(yz / unsigned(ny));
    const int y1 = wrapm(y + 1, ny), z1 = wrapm(z + 1, d.nz);
    const size_t r00 = (size_t(y) + size_t(ny) * z) * nx, r10 = (size_t(y1) + size_t(ny) * z) * nx;
    const size_t r01 = (size_t(y) + size_t(ny) * z1) * nx, r11 = (size_t(y1) + size_t(ny) * z1) * nx;
    float F[3][4];
    face_wht(chi, nv, r00 + x0, r10 + x0, r01 + x0, r11 + x0, F);
#pragma unroll
    for (int i = 0; i < kRun; i++) {
      const int x = x0 + i;
      if (x < nx) {
        const int xn = x + 1 < nx ? x + 1 : 0;
        float G[3][4];
        face_wht(chi, nv, r00 + xn, r10 + xn, r01 + xn, r11 + xn, G);
        float w[3][8];
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
          for (int q = 0; q < 4; q++) {
            w[c][2 * q] = dw[c][2 * q] - (F[c][q] + G[c][q]);
            w[c][2 * q + 1] = dw[c][2 * q + 1] - (F[c][q] - G[c][q]);
          }
        float E[6];
        int cnt = 0;
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
          for (int bq = a; bq < 3; bq++) {
            const float* u = w[a];
            const float* t = w[bq];
            const float s1 = u[1] * t[1] + u[2] * t[2] + u[4] * t[4];
            const float s2 = u[3] * t[3] + u[5] * t[5] + u[6] * t[6];
            E[cnt++] = l0 * (u[0] * t[0]) + l1 * s1 + l2 * s2 + l3 * (u[7] * t[7]);
          }
        const size_t e = size_t(yz) * nx + x;
        if (kKH) {
          const double k = __ldg(ks + e);
#pragma unroll
          for (int j = 0; j < 6; j++) v[j] += k * double(E[j]);
        }
        if (kSens) {
          float sv = 0.f;
#pragma unroll
          for (int j = 0; j < 6; j++) sv += E[j] * sw.w[j];
          const float pr = (p == 1.f) ? 1.f : p * powf(__ldg(kraw + e), p - 1.f);
          sens[size_t(yz) * pitchT + x] = sv * pr;
        }
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
          for (int q = 0; q < 4; q++) F[c][q] = G[c][q];
      }
    }
    // the pitch padding of the row, by the thread of its last run
    if (kSens && x0 + kRun >= nx)
      for (int x = nx; x < pitchT; x++) sens[size_t(yz) * pitchT + x] = 0.f;
  }
  if (kKH) {
    block_reduce_f64<6>(v, smem);
    if (threadIdx.x == 0)
#pragma unroll
      for (int i = 0; i < 6; i++) partials[blockIdx.x * 6 + i] = v[i];
    if (last_block(&sc->counter[T_KH])) {
      double t[6];
      reduce_partials<6>(partials, gridDim.x, t, smem);
      if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < 6; i++) sc->kh[i] = t[i];
        sc->counter[T_KH] = 0;
      }
    }
  }
}

// 6 unpitched fields of dK^H_ab / dk_e.
static __global__ void __launch_bounds__(kBlock) k_energy_fields(Dims d, const float* __restrict__ chi, FineOp op,
                                                          ElemFields ef, float* __restrict__ out) {
  const size_t nv = d.nv();
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= nv) return;
  float E[6];
  elem_energy(d, e, chi, op, ef, E);
#pragma unroll
  for (int i = 0; i < 6; i++) out[i * nv + e] = E[i];
}

}  // namespace otm
