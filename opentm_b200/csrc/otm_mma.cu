// otm_mma.cu -- method of moving asymptotes in FP64 on the device (Svanberg's MMA with the
// primal-dual interior-point subsolver), replacing MMAOptimizer / mmasubDevice
// (optimization/mmaOptimizer.cu:18-78, optimization/mmaOpt.cu:429-1062, mmaOpt.cpp:38-73).
//
// Every pass over the n design variables is one kernel that also reduces what the next step
// needs (sums with a fixed-order last-block finalisation, maxima). A Newton step is two passes:
// the step bounds of the direction, then the line-search trial, which recomputes the direction,
// writes the trial point to spare arrays and reduces both the residual there and the next Newton
// system (accepting the step swaps the arrays). The (m+1) x (m+1) KKT system (m <= 8) is solved
// in FP64 on the host, where the reference used Eigen.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "opentm_b200_mma.h"
#include "otm_common.cuh"
#include "otm_mg_kernels.cuh"

namespace otm {

constexpr int kMmaMaxM = OTM_MMA_MAX_CONSTRAINTS;
constexpr double kEpsiMin = 1e-7, kRaa0 = 1e-5, kAlbefa = 0.1, kAsyInit = 0.5, kAsyIncr = 1.2, kAsyDecr = 0.7;

struct MVec {
  double v[kMmaMaxM];
};

// Work arrays of one subsolve, n (or m * n) doubles each. dx, dxsi, deta hold the line search's
// trial point, which trades places with xs, xsi, eta when it is accepted.
struct MmaWork {
  size_t n = 0;
  int m = 0;
  double *alfa = nullptr, *beta = nullptr, *p0 = nullptr, *q0 = nullptr, *P = nullptr, *Q = nullptr;
  double *xs = nullptr, *xsi = nullptr, *eta = nullptr, *dx = nullptr, *dxsi = nullptr, *deta = nullptr;
  double* partials = nullptr;  // kMaxPartials * 96
  double* result = nullptr;    // 96
  unsigned int* counter = nullptr;
  double* host = nullptr;      // pinned, 96
};

constexpr int kMmaSlots = 128;  // >= 2 + 3 m + m^2 for m <= 8

template <int NM>
__device__ __forceinline__ void block_reduce_max(double (&v)[NM], double* smem) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < NM; i++)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[i] = fmax(v[i], __shfl_down_sync(0xffffffffu, v[i], off));
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < NM; i++) smem[warp * NM + i] = v[i];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NM; i++) {
      double x = lane < nwarps ? smem[lane * NM + i] : -1e300;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) x = fmax(x, __shfl_down_sync(0xffffffffu, x, off));
      v[i] = x;
    }
  }
}

// Block partials of NS sums and NM maxima, then the last block writes result[0..NS+NM).
template <int NS, int NM>
__device__ __forceinline__ void reduce_to_result(double (&s)[NS], double (&mx)[NM], double* partials,
                                                 double* result, unsigned int* counter) {
  __shared__ double smem[32 * (NS > NM ? NS : NM)];
  block_reduce_f64<NS>(s, smem);
  block_reduce_max<NM>(mx, smem);
  constexpr int W = NS + NM;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NS; i++) partials[blockIdx.x * W + i] = s[i];
#pragma unroll
    for (int i = 0; i < NM; i++) partials[blockIdx.x * W + NS + i] = mx[i];
  }
  if (last_block(counter)) {
    // one warp per value: lanes stride over the blocks, then a shuffle reduction (fixed order)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = warp; i < W; i += int(blockDim.x >> 5)) {
      double acc = i < NS ? 0.0 : -1e300;
#pragma unroll 8
      for (int b = lane; b < int(gridDim.x); b += 32) {
        const double v = __ldcg(partials + b * W + i);  // L2: never a stale L1 line
        acc = i < NS ? acc + v : fmax(acc, v);
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double o = __shfl_xor_sync(0xffffffffu, acc, off);
        acc = i < NS ? acc + o : fmax(acc, o);
      }
      if (lane == 0) result[i] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) *counter = 0;
  }
}

// Asymptotes, move limits, approximation coefficients p0, q0, P, Q, the constraint offsets
// sum_j P/ux + Q/xl, and the subsolver's starting point (mmasub_ker, optimization/mmaOpt.cu:834-1019).
template <int M>
__global__ void __launch_bounds__(256) k_mma_setup(size_t n, int itn, const double* __restrict__ xvar,
                                                   const double* __restrict__ xmin, const double* __restrict__ xmax,
                                                   const double* __restrict__ xold1,
                                                   const double* __restrict__ xold2, const double* __restrict__ df0dx,
                                                   const double* __restrict__ dgdx, size_t ldg, double* low,
                                                   double* upp, double move, MmaWork w) {
  double bs[M];
  double dummy[1] = {-1e300};
#pragma unroll
  for (int i = 0; i < M; i++) bs[i] = 0.0;
  for (size_t j = size_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += size_t(gridDim.x) * blockDim.x) {
    const double x = xvar[j], dxr = xmax[j] - xmin[j];
    double lo, up;
    if (itn <= 2) {
      lo = x - kAsyInit * dxr;
      up = x + kAsyInit * dxr;
    } else {
      const double zzz = (x - xold1[j]) * (xold1[j] - xold2[j]);
      const double f = zzz > 0 ? kAsyIncr : (zzz < 0 ? kAsyDecr : 1.0);
      lo = x - f * (xold1[j] - low[j]);
      up = x + f * (upp[j] - xold1[j]);
      lo = fmin(fmax(lo, x - 10.0 * dxr), x - 0.01 * dxr);
      up = fmax(fmin(up, x + 10.0 * dxr), x + 0.01 * dxr);
    }
    low[j] = lo;
    upp[j] = up;
    const double al = fmax(fmax(lo + kAlbefa * (x - lo), x - move * dxr), xmin[j]);
    const double be = fmin(fmin(up - kAlbefa * (up - x), x + move * dxr), xmax[j]);
    w.alfa[j] = al;
    w.beta[j] = be;
    const double xmamiinv = 1.0 / fmax(dxr, 1e-5);
    const double ux1 = up - x, xl1 = x - lo, ux2 = ux1 * ux1, xl2 = xl1 * xl1;
    const double dp = fmax(df0dx[j], 0.0), dm = fmax(-df0dx[j], 0.0);
    const double pq0 = 1e-3 * (dp + dm) + kRaa0 * xmamiinv;
    w.p0[j] = (dp + pq0) * ux2;
    w.q0[j] = (dm + pq0) * xl2;
#pragma unroll
    for (int i = 0; i < M; i++) {
      const double g = dgdx[i * ldg + j];
      const double pp = fmax(g, 0.0), qq = fmax(-g, 0.0);
      const double pq = 1e-3 * (pp + qq) + kRaa0 * xmamiinv;
      const double Pij = (pp + pq) * ux2, Qij = (qq + pq) * xl2;
      w.P[i * n + j] = Pij;
      w.Q[i * n + j] = Qij;
      bs[i] += Pij / ux1 + Qij / xl1;
    }
    const double xs = 0.5 * (al + be);
    w.xs[j] = xs;
    w.xsi[j] = fmax(1.0 / (xs - al), 1.0);
    w.eta[j] = fmax(1.0 / (be - xs), 1.0);
    w.dx[j] = 0.0;
    w.dxsi[j] = 0.0;
    w.deta[j] = 0.0;
  }
  reduce_to_result<M, 1>(bs, dummy, w.partials, w.result, w.counter);
}

// The per-variable data a subsolver pass reads: the point, its bounds and the approximation.
template <int M>
struct MmaElem {
  double x, xsi, eta, low, upp, al, be, p0, q0, P[M], Q[M];
};

template <int M>
__device__ __forceinline__ void load_elem(const MmaWork& w, const double* __restrict__ low,
                                          const double* __restrict__ upp, size_t j, MmaElem<M>& e) {
  e.x = w.xs[j];
  e.xsi = w.xsi[j];
  e.eta = w.eta[j];
  e.low = low[j];
  e.upp = upp[j];
  e.al = w.alfa[j];
  e.be = w.beta[j];
  e.p0 = w.p0[j];
  e.q0 = w.q0[j];
#pragma unroll
  for (int i = 0; i < M; i++) {
    e.P[i] = w.P[i * w.n + j];
    e.Q[i] = w.Q[i * w.n + j];
  }
}

// Elements j and j + 1 (j even; n even and every array 16-byte aligned): one 16-byte load per
// array, twice the bytes in flight per instruction.
template <int M>
__device__ __forceinline__ void load_pair(const MmaWork& w, const double* __restrict__ low,
                                          const double* __restrict__ upp, size_t j, MmaElem<M>& a, MmaElem<M>& b) {
  auto ld = [j](const double* p, double& u, double& v) {
    const double2 t = *reinterpret_cast<const double2*>(p + j);
    u = t.x;
    v = t.y;
  };
  ld(w.xs, a.x, b.x);
  ld(w.xsi, a.xsi, b.xsi);
  ld(w.eta, a.eta, b.eta);
  ld(low, a.low, b.low);
  ld(upp, a.upp, b.upp);
  ld(w.alfa, a.al, b.al);
  ld(w.beta, a.be, b.be);
  ld(w.p0, a.p0, b.p0);
  ld(w.q0, a.q0, b.q0);
#pragma unroll
  for (int i = 0; i < M; i++) {
    ld(w.P + i * w.n, a.P[i], b.P[i]);
    ld(w.Q + i * w.n, a.Q[i], b.Q[i]);
  }
}

// Newton direction of x, xsi, eta at e for multiplier lam and its step dlam (subsolv's dx, dxsi,
// deta, optimization/mmaOpt.cu:429-830), shared by the two passes below so both see the same
// values without storing them. The five distinct denominators are inverted once.
template <int M>
__device__ __forceinline__ void mma_dir(const MmaElem<M>& e, const MVec& lam, const MVec& dlam, double epsi,
                                        double* dx, double* dxsi, double* deta, double* rxa_out, double* rbx_out) {
  const double x = e.x;
  const double rux = 1.0 / (e.upp - x), rxl = 1.0 / (x - e.low);
  const double rux2 = rux * rux, rxl2 = rxl * rxl;
  const double rxa = 1.0 / (x - e.al), rbx = 1.0 / (e.be - x);
  double plam = e.p0, qlam = e.q0, gl = 0.0;
#pragma unroll
  for (int i = 0; i < M; i++) {
    plam += e.P[i] * lam.v[i];
    qlam += e.Q[i] * lam.v[i];
    gl += (e.P[i] * rux2 - e.Q[i] * rxl2) * dlam.v[i];
  }
  const double dpsidx = plam * rux2 - qlam * rxl2;
  const double delx = dpsidx - epsi * rxa + epsi * rbx;
  const double diagx = 2.0 * (plam * rux2 * rux + qlam * rxl2 * rxl) + e.xsi * rxa + e.eta * rbx;
  const double rd = 1.0 / diagx;
  *dx = -(delx + gl) * rd;
  *dxsi = -e.xsi + epsi * rxa - e.xsi * *dx * rxa;
  *deta = -e.eta + epsi * rbx + e.eta * *dx * rbx;
  *rxa_out = rxa;
  *rbx_out = rbx;
}

// The line search's step bounds: the largest ratios -1.01 dxsi/xsi, -1.01 deta/eta,
// -1.01 dx/(x - alfa), 1.01 dx/(beta - x), without storing the direction (the trial pass
// recomputes it). VW consecutive variables per loop step.
template <int M, int VW>
__global__ void __launch_bounds__(256) k_mma_dirmax(MVec lam, MVec dlam, double epsi, const double* __restrict__ low,
                                                    const double* __restrict__ upp, MmaWork w) {
  double s[1] = {0.0};
  double mx[4] = {-1e300, -1e300, -1e300, -1e300};
  const size_t nq = w.n / VW;
  for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nq; q += size_t(gridDim.x) * blockDim.x) {
    MmaElem<M> e[VW];
    if (VW == 2)
      load_pair<M>(w, low, upp, 2 * q, e[0], e[VW - 1]);
    else
      load_elem<M>(w, low, upp, q, e[0]);
#pragma unroll
    for (int v = 0; v < VW; v++) {
      double dx, dxsi, deta, rxa, rbx;
      mma_dir<M>(e[v], lam, dlam, epsi, &dx, &dxsi, &deta, &rxa, &rbx);
      mx[0] = fmax(mx[0], -1.01 * dxsi / e[v].xsi);
      mx[1] = fmax(mx[1], -1.01 * deta / e[v].eta);
      mx[2] = fmax(mx[2], -1.01 * dx * rxa);
      mx[3] = fmax(mx[3], 1.01 * dx * rbx);
    }
  }
  reduce_to_result<1, 4>(s, mx, w.partials, w.result, w.counter);
}

// One pass at the trial point x + steg dx (steg = 0: the committed point, nothing written): the
// relaxed KKT residual with the trial multiplier lam ([sum of squares, max |.|] of the n-part and
// gvec_i = sum_j P/ux + Q/xl) and, at the same point, the pieces of the next Newton system (gvec,
// GG delx/diagx, GG diag(1/diagx) GG^T), so an accepted step needs no further pass. The trial
// point goes to xs_out / xsi_out / eta_out; accepting it is a pointer swap. VW consecutive
// variables per loop step.
// result = [resid sum of squares, resid gvec (M), newton gvec (M), GG delx/diagx (M),
//           GG diag(1/diagx) GG^T (M*M), resid max |.|].
template <int M, int VW>
__global__ void __launch_bounds__(256) k_mma_trial(double steg, MVec lam, MVec lam_dir, MVec dlam, double epsi,
                                                   double epsi_dir, const double* __restrict__ low,
                                                   const double* __restrict__ upp, double* xs_out, double* xsi_out,
                                                   double* eta_out, MmaWork w) {
  constexpr int NS = 1 + M + M + M + M * M;
  double s[NS];
  double mx[1] = {0.0};
#pragma unroll
  for (int i = 0; i < NS; i++) s[i] = 0.0;
  const size_t nq = w.n / VW;
  for (size_t q = size_t(blockIdx.x) * blockDim.x + threadIdx.x; q < nq; q += size_t(gridDim.x) * blockDim.x) {
    MmaElem<M> e[VW];
    if (VW == 2)
      load_pair<M>(w, low, upp, 2 * q, e[0], e[VW - 1]);
    else
      load_elem<M>(w, low, upp, q, e[0]);
#pragma unroll
    for (int v = 0; v < VW; v++) {
      if (steg != 0.0) {
        double dx, dxsi, deta, r0, r1;
        mma_dir<M>(e[v], lam_dir, dlam, epsi_dir, &dx, &dxsi, &deta, &r0, &r1);
        e[v].x = e[v].x + steg * dx;
        e[v].xsi = e[v].xsi + steg * dxsi;
        e[v].eta = e[v].eta + steg * deta;
      }
      const double x = e[v].x, xsi = e[v].xsi, eta = e[v].eta, al = e[v].al, be = e[v].be;
      // residual
      const double uxi = 1.0 / (e[v].upp - x), xli = 1.0 / (x - e[v].low);
      double plam = e[v].p0, qlam = e[v].q0;
#pragma unroll
      for (int i = 0; i < M; i++) {
        plam += e[v].P[i] * lam.v[i];
        qlam += e[v].Q[i] * lam.v[i];
        s[1 + i] += e[v].P[i] * uxi + e[v].Q[i] * xli;
      }
      const double rex = plam * uxi * uxi - qlam * xli * xli - xsi + eta;
      const double rexsi = xsi * (x - al) - epsi;
      const double reeta = eta * (be - x) - epsi;
      s[0] += rex * rex + rexsi * rexsi + reeta * reeta;
      mx[0] = fmax(mx[0], fmax(fabs(rex), fmax(fabs(rexsi), fabs(reeta))));
      // Newton system pieces (its gvec is the residual's), with the reciprocals above and of
      // x - alfa, beta - x, diagx
      const double rux2 = uxi * uxi, rxl2 = xli * xli;
      const double rxa = 1.0 / (x - al), rbx = 1.0 / (be - x);
      double GG[M];
#pragma unroll
      for (int i = 0; i < M; i++) GG[i] = e[v].P[i] * rux2 - e[v].Q[i] * rxl2;
      const double dpsidx = plam * rux2 - qlam * rxl2;
      const double delx = dpsidx - epsi * rxa + epsi * rbx;
      const double diagx = 2.0 * (plam * rux2 * uxi + qlam * rxl2 * xli) + xsi * rxa + eta * rbx;
      const double id = 1.0 / diagx, dd = delx * id;
#pragma unroll
      for (int i = 0; i < M; i++) {
        s[1 + 2 * M + i] += GG[i] * dd;
#pragma unroll
        for (int k = 0; k < M; k++) s[1 + 3 * M + i * M + k] += GG[i] * GG[k] * id;
      }
    }
    if (steg != 0.0) {
      if (VW == 2) {
        const size_t j = 2 * q;
        *reinterpret_cast<double2*>(xs_out + j) = make_double2(e[0].x, e[VW - 1].x);
        *reinterpret_cast<double2*>(xsi_out + j) = make_double2(e[0].xsi, e[VW - 1].xsi);
        *reinterpret_cast<double2*>(eta_out + j) = make_double2(e[0].eta, e[VW - 1].eta);
      } else {
        xs_out[q] = e[0].x;
        xsi_out[q] = e[0].xsi;
        eta_out[q] = e[0].eta;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < M; i++) s[1 + M + i] = s[1 + i];
  reduce_to_result<NS, 1>(s, mx, w.partials, w.result, w.counter);
}

__global__ void k_mma_finish(size_t n, double* xvar, double* xold1, double* xold2, const double* xs) {
  for (size_t j = size_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += size_t(gridDim.x) * blockDim.x) {
    xold2[j] = xold1[j];
    xold1[j] = xvar[j];
    xvar[j] = xs[j];
  }
}

__global__ void k_cast_f2d(size_t n, const float* __restrict__ a, double* b) {
  for (size_t j = size_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += size_t(gridDim.x) * blockDim.x)
    b[j] = double(a[j]);
}

__global__ void k_cast_d2f(size_t n, const double* __restrict__ a, float* b) {
  for (size_t j = size_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += size_t(gridDim.x) * blockDim.x)
    b[j] = float(a[j]);
}

__global__ void k_fill(size_t n, double v, double* a) {
  for (size_t j = size_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += size_t(gridDim.x) * blockDim.x) a[j] = v;
}

// Dense (m+1) x (m+1) solve with partial pivoting (replaces Eigen ColPivHouseholderQR,
// optimization/mmaOpt.cpp:48-73).
static bool dense_solve(int n, std::vector<double> A, std::vector<double>& b) {
  for (int k = 0; k < n; k++) {
    int p = k;
    for (int i = k + 1; i < n; i++)
      if (std::fabs(A[i * n + k]) > std::fabs(A[p * n + k])) p = i;
    if (A[p * n + k] == 0.0) return false;
    if (p != k) {
      for (int j = 0; j < n; j++) std::swap(A[k * n + j], A[p * n + j]);
      std::swap(b[k], b[p]);
    }
    for (int i = k + 1; i < n; i++) {
      const double l = A[i * n + k] / A[k * n + k];
      for (int j = k; j < n; j++) A[i * n + j] -= l * A[k * n + j];
      b[i] -= l * b[k];
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = b[i];
    for (int j = i + 1; j < n; j++) s -= A[i * n + j] * b[j];
    b[i] = s / A[i * n + i];
  }
  return true;
}

static otm_status work_alloc(MmaWork& w, int m, size_t n, cudaStream_t s, bool async) {
  w.m = m;
  w.n = n;
  double** arr[] = {&w.alfa, &w.beta, &w.p0, &w.q0, &w.xs, &w.xsi, &w.eta, &w.dx, &w.dxsi, &w.deta};
  for (double** a : arr) {
    if (async)
      OTM_CUDA(scratch_malloc((void**)a, n * sizeof(double), s));
    else
      OTM_CUDA(cudaMalloc((void**)a, n * sizeof(double)));
  }
  for (double** a : {&w.P, &w.Q}) {
    if (async)
      OTM_CUDA(scratch_malloc((void**)a, size_t(m) * n * sizeof(double), s));
    else
      OTM_CUDA(cudaMalloc((void**)a, size_t(m) * n * sizeof(double)));
  }
  const size_t small = size_t(kMaxPartials) * kMmaSlots * sizeof(double) + kMmaSlots * sizeof(double) + 64;
  char* buf = nullptr;
  if (async)
    OTM_CUDA(scratch_malloc((void**)&buf, small, s));
  else
    OTM_CUDA(cudaMalloc((void**)&buf, small));
  w.partials = (double*)buf;
  w.result = w.partials + size_t(kMaxPartials) * kMmaSlots;
  w.counter = (unsigned int*)(w.result + kMmaSlots);
  OTM_CUDA(cudaMemsetAsync(w.counter, 0, 64, s));
  OTM_CUDA(cudaMallocHost((void**)&w.host, kMmaSlots * sizeof(double)));
  return OTM_OK;
}

static void work_free(MmaWork& w, cudaStream_t s, bool async) {
  double* arr[] = {w.alfa, w.beta, w.p0, w.q0, w.xs, w.xsi, w.eta, w.dx, w.dxsi, w.deta, w.P, w.Q, w.partials};
  for (double* a : arr)
    if (a) {
      if (async)
        cudaFreeAsync(a, s);
      else
        cudaFree(a);
    }
  if (w.host) cudaFreeHost(w.host);
  w = MmaWork{};
}

// Dispatch on the (compile-time) constraint count.
template <template <int> class K, typename... Args>
static void dispatch_m(int m, Args&&... args) {
  switch (m) {
    case 1: K<1>::run(args...); break;
    case 2: K<2>::run(args...); break;
    case 3: K<3>::run(args...); break;
    case 4: K<4>::run(args...); break;
    case 5: K<5>::run(args...); break;
    case 6: K<6>::run(args...); break;
    case 7: K<7>::run(args...); break;
    default: K<8>::run(args...); break;
  }
}

template <int M>
struct LaunchSetup {
  static void run(int nb, cudaStream_t s, size_t n, int itn, const double* xvar, const double* xmin,
                  const double* xmax, const double* xold1, const double* xold2, const double* df0dx,
                  const double* dgdx, size_t ldg, double* low, double* upp, double move, MmaWork w) {
    k_mma_setup<M><<<nb, 256, 0, s>>>(n, itn, xvar, xmin, xmax, xold1, xold2, df0dx, dgdx, ldg, low, upp, move, w);
  }
};

template <int M>
struct LaunchDirmax {
  static void run(int nb, bool pairs, cudaStream_t s, MVec lam, MVec dlam, double epsi, const double* low,
                  const double* upp, MmaWork w) {
    if (pairs)
      k_mma_dirmax<M, 2><<<nb, 256, 0, s>>>(lam, dlam, epsi, low, upp, w);
    else
      k_mma_dirmax<M, 1><<<nb, 256, 0, s>>>(lam, dlam, epsi, low, upp, w);
  }
};
template <int M>
struct LaunchTrial {
  static void run(int nb, bool pairs, cudaStream_t s, double steg, MVec lam, MVec lam_dir, MVec dlam, double epsi,
                  double epsi_dir, const double* low, const double* upp, double* xo, double* xsio, double* etao,
                  MmaWork w) {
    if (pairs)
      k_mma_trial<M, 2><<<nb, 256, 0, s>>>(steg, lam, lam_dir, dlam, epsi, epsi_dir, low, upp, xo, xsio, etao, w);
    else
      k_mma_trial<M, 1><<<nb, 256, 0, s>>>(steg, lam, lam_dir, dlam, epsi, epsi_dir, low, upp, xo, xsio, etao, w);
  }
};

static otm_status fetch(MmaWork& w, cudaStream_t s, int count) {
  OTM_CUDA(cudaMemcpyAsync(w.host, w.result, count * sizeof(double), cudaMemcpyDeviceToHost, s));
  OTM_CUDA(cudaStreamSynchronize(s));
  return OTM_OK;
}

// One MMA step (mmasub_g, optimization/mmaOpt.cu:1021-1062): device arrays, host-side a/c/d/gval.
static otm_status mmasub_run(cudaStream_t s, int m, size_t n, int itn, double* xvar, const double* xmin,
                             const double* xmax, double* xold1, double* xold2, const double* df0dx,
                             const double* gval, const double* dgdx, size_t ldg, double* low, double* upp,
                             double a0, const double* a, const double* c, const double* d, double move, MmaWork& w,
                             uint64_t* launches) {
  const int nb = int(std::min<size_t>(kMaxPartials, std::max<size_t>(1, (n + 255) / 256)));
  uint64_t L = 0;
  dispatch_m<LaunchSetup>(m, nb, s, n, itn, xvar, xmin, xmax, xold1, xold2, df0dx, dgdx, ldg, low, upp, move, w);
  L++;
  OTM_CHECK_LAUNCH("k_mma_setup");
  OTM_TRY(fetch(w, s, m));
  std::vector<double> b(m);
  for (int i = 0; i < m; i++) b[i] = w.host[i] - gval[i];

  // subsolv (optimization/mmaOpt.cu:429-830): dual/slack variables of size m live on the host
  std::vector<double> y(m, 1.0), lam(m, 1.0), mu(m), sv(m, 1.0);
  for (int i = 0; i < m; i++) mu[i] = std::max(0.5 * c[i], 1.0);
  double z = 1.0, zet = 1.0, epsi = 1.0;
  MVec lamv{}, dlamv{};
  std::vector<double> gvec(m);

  auto m_residual = [&](const std::vector<double>& yy, double zz, const std::vector<double>& ll,
                        const std::vector<double>& mm, double ze, const std::vector<double>& ss, double* n2,
                        double* mxv) {
    double ad = 0.0;
    for (int i = 0; i < m; i++) ad += a[i] * ll[i];
    auto acc = [&](double r) {
      *n2 += r * r;
      *mxv = std::max(*mxv, std::fabs(r));
    };
    for (int i = 0; i < m; i++) acc(c[i] + d[i] * yy[i] - mm[i] - ll[i]);
    acc(a0 - ze - ad);
    for (int i = 0; i < m; i++) acc(gvec[i] - a[i] * zz - yy[i] + ss[i] - b[i]);
    for (int i = 0; i < m; i++) acc(mm[i] * yy[i] - epsi);
    acc(ze * zz - epsi);
    for (int i = 0; i < m; i++) acc(ll[i] * ss[i] - epsi);
  };
  // One pass at x + steg * (direction for lam_dir, dlam): residual norm / max with the trial
  // multipliers, and the Newton pieces there (cached in newt: gvec, GG delx/diagx, GG GG^T/diagx).
  // With steg != 0 the trial point is written to the spare arrays w.dx, w.dxsi, w.deta.
  const int NS = 1 + 3 * m + m * m;
  // pairs of variables per loop step when every array the passes read is 16-byte aligned at
  // every row (n even; the work arrays come from the allocator, low and upp from the caller)
  // (m <= 4: beyond that the pair of elements no longer fits the registers)
  const bool pairs = m <= 4 && n % 2 == 0 && (reinterpret_cast<uintptr_t>(low) % 16) == 0 &&
                     (reinterpret_cast<uintptr_t>(upp) % 16) == 0;
  const int nbp = int(std::min<size_t>(kMaxPartials, std::max<size_t>(1, (n / (pairs ? 2 : 1) + 255) / 256)));
  std::vector<double> newt(size_t(2 * m + m * m));
  auto trial = [&](double steg, const std::vector<double>& yy, double zz, const std::vector<double>& ll,
                   const std::vector<double>& mm, double ze, const std::vector<double>& ss,
                   const std::vector<double>& ldir, const MVec& dl, double* nrm, double* mxv) -> otm_status {
    MVec lt{}, ld{};
    for (int i = 0; i < m; i++) {
      lt.v[i] = ll[i];
      ld.v[i] = ldir[i];
    }
    dispatch_m<LaunchTrial>(m, nbp, pairs, s, steg, lt, ld, dl, epsi, epsi, (const double*)low, (const double*)upp,
                            w.dx, w.dxsi, w.deta, w);
    L++;
    OTM_CHECK_LAUNCH("k_mma_trial");
    OTM_TRY(fetch(w, s, NS + 1));
    double n2 = w.host[0], mx = w.host[NS];
    for (int i = 0; i < m; i++) gvec[i] = w.host[1 + i];
    for (size_t i = 0; i < newt.size(); i++) newt[i] = w.host[1 + m + i];
    m_residual(yy, zz, ll, mm, ze, ss, &n2, &mx);
    *nrm = std::sqrt(n2);
    *mxv = mx;
    return OTM_OK;
  };
  // the trial point becomes the committed one (the work arrays keep owning both sets)
  auto accept = [&]() {
    std::swap(w.xs, w.dx);
    std::swap(w.xsi, w.dxsi);
    std::swap(w.eta, w.deta);
  };

  std::vector<double> dy(m), dmu(m), ds(m), dl(m), yo(m), lo(m), muo(m), so(m);
  while (epsi > kEpsiMin) {
    double residunorm, residumax;
    OTM_TRY(trial(0.0, y, z, lam, mu, zet, sv, lam, dlamv, &residunorm, &residumax));
    int ittt = 0;
    while (residumax > 0.9 * epsi && ittt < 200) {
      ittt++;
      for (int i = 0; i < m; i++) lamv.v[i] = lam[i];
      const double* hn = newt.data();  // Newton pieces at the committed point
      for (int i = 0; i < m; i++) gvec[i] = hn[i];
      double adl = 0.0;
      for (int i = 0; i < m; i++) adl += a[i] * lam[i];
      const double delz = a0 - adl - epsi / z;
      std::vector<double> AA(size_t(m + 1) * (m + 1), 0.0), bb(m + 1);
      std::vector<double> dely(m), diagy(m);
      for (int i = 0; i < m; i++) {
        dely[i] = c[i] + d[i] * y[i] - lam[i] - epsi / y[i];
        const double dellam = gvec[i] - a[i] * z - y[i] - b[i] + epsi / lam[i];
        diagy[i] = d[i] + mu[i] / y[i];
        bb[i] = dellam + dely[i] / diagy[i] - hn[m + i];
        for (int k = 0; k < m; k++) AA[size_t(i) * (m + 1) + k] = hn[2 * m + i * m + k];
        AA[size_t(i) * (m + 1) + i] += sv[i] / lam[i] + 1.0 / diagy[i];
        AA[size_t(i) * (m + 1) + m] = a[i];
        AA[size_t(m) * (m + 1) + i] = a[i];
      }
      AA[size_t(m) * (m + 1) + m] = -zet / z;
      bb[m] = delz;
      if (!dense_solve(m + 1, AA, bb)) {
        set_error("singular MMA Newton system");
        return OTM_ERR_NAN;
      }
      for (int i = 0; i < m; i++) dl[i] = bb[i];
      const double dz = bb[m];
      for (int i = 0; i < m; i++) {
        dy[i] = -dely[i] / diagy[i] + dl[i] / diagy[i];
        dmu[i] = -mu[i] + epsi / y[i] - (mu[i] * dy[i]) / y[i];
        ds[i] = -sv[i] + epsi / lam[i] - (sv[i] * dl[i]) / lam[i];
        dlamv.v[i] = dl[i];
      }
      const double dzet = -zet + epsi / z - zet * dz / z;
      dispatch_m<LaunchDirmax>(m, nbp, pairs, s, lamv, dlamv, epsi, (const double*)low, (const double*)upp, w);
      L++;
      OTM_CHECK_LAUNCH("k_mma_dirmax");
      OTM_TRY(fetch(w, s, 5));
      double stm = std::max(w.host[1], w.host[2]);  // xsi, eta parts
      for (int i = 0; i < m; i++) {
        stm = std::max(stm, -1.01 * dy[i] / y[i]);
        stm = std::max(stm, -1.01 * dl[i] / lam[i]);
        stm = std::max(stm, -1.01 * dmu[i] / mu[i]);
        stm = std::max(stm, -1.01 * ds[i] / sv[i]);
      }
      stm = std::max(stm, -1.01 * dz / z);
      stm = std::max(stm, -1.01 * dzet / zet);
      const double stmalbe = std::max(w.host[3], w.host[4]);
      double steg = 1.0 / std::max(std::max(stmalbe, stm), 1.0);
      if (std::isnan(steg)) {
        set_error("NaN step in the MMA subproblem");
        return OTM_ERR_NAN;
      }
      yo = y;
      lo = lam;
      muo = mu;
      so = sv;
      const double zo = z, zeto = zet;
      int itto = 0;
      double resinew = 2 * residunorm, resimax = residumax;
      while (resinew > residunorm && itto < 50) {
        itto++;
        for (int i = 0; i < m; i++) {
          y[i] = yo[i] + steg * dy[i];
          lam[i] = lo[i] + steg * dl[i];
          mu[i] = muo[i] + steg * dmu[i];
          sv[i] = so[i] + steg * ds[i];
        }
        z = zo + steg * dz;
        zet = zeto + steg * dzet;
        OTM_TRY(trial(steg, y, z, lam, mu, zet, sv, lo, dlamv, &resinew, &resimax));
        steg /= 2;
      }
      accept();  // the last point tried, as the reference commits after its line search
      residunorm = resinew;
      residumax = resimax;
    }
    epsi *= 0.1;
  }
  k_mma_finish<<<nb, 256, 0, s>>>(n, xvar, xold1, xold2, w.xs);
  L++;
  OTM_CHECK_LAUNCH("k_mma_finish");
  if (launches) *launches += L;
  count_launches(L);
  return OTM_OK;
}

}  // namespace otm

using namespace otm;

struct otm_mma {
  int m = 0;
  size_t n = 0;
  double a0 = 1.0;
  std::vector<double> a, c, d;
  cudaStream_t stream = nullptr;
  double *xvar = nullptr, *xmin = nullptr, *xmax = nullptr, *xold1 = nullptr, *xold2 = nullptr;
  double *low = nullptr, *upp = nullptr, *df0dx = nullptr, *dgdx = nullptr;
  MmaWork w;
  ~otm_mma() {
    double* arr[] = {xvar, xmin, xmax, xold1, xold2, low, upp, df0dx, dgdx};
    for (double* p : arr)
      if (p) cudaFree(p);
    work_free(w, nullptr, false);
  }
};

extern "C" {

otm_status otm_mma_create(int m, int n, double a0, double a, double c, double d, otm_mma** out) {
  if (!out || m < 1 || m > kMmaMaxM || n < 1) {
    set_error("need 1 <= m <= 8 constraints and n >= 1 variables");
    return OTM_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  otm_mma* o = new (std::nothrow) otm_mma();
  if (!o) return OTM_ERR_OUT_OF_MEMORY;
  o->m = m;
  o->n = size_t(n);
  o->a0 = a0;
  o->a.assign(m, a);
  o->c.assign(m, c);
  o->d.assign(m, d);
  auto fail = [&](otm_status st) {
    delete o;
    return st;
  };
  double** arr[] = {&o->xvar, &o->xmin, &o->xmax, &o->xold1, &o->xold2, &o->low, &o->upp, &o->df0dx};
  for (double** p : arr) {
    cudaError_t e = cudaMalloc((void**)p, o->n * sizeof(double));
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc"));
    cudaMemset(*p, 0, o->n * sizeof(double));
  }
  cudaError_t e = cudaMalloc((void**)&o->dgdx, size_t(m) * o->n * sizeof(double));
  if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc"));
  otm_status st = work_alloc(o->w, m, o->n, nullptr, false);
  if (st != OTM_OK) return fail(st);
  if (cudaDeviceSynchronize() != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "otm_mma_create"));
  *out = o;
  return OTM_OK;
}

otm_status otm_mma_destroy(otm_mma* mma) {
  if (!mma) return OTM_ERR_INVALID_ARGUMENT;
  cudaStreamSynchronize(mma->stream);
  delete mma;
  return OTM_OK;
}

otm_status otm_mma_set_stream(otm_mma* mma, void* stream) {
  if (!mma) return OTM_ERR_INVALID_ARGUMENT;
  mma->stream = (cudaStream_t)stream;
  return OTM_OK;
}

otm_status otm_mma_set_bound_scalar(otm_mma* mma, float xmin, float xmax) {
  if (!mma || !(xmax >= xmin)) return OTM_ERR_INVALID_ARGUMENT;
  const int nb = int(std::min<size_t>(kMaxPartials, (mma->n + 255) / 256));
  k_fill<<<nb, 256, 0, mma->stream>>>(mma->n, double(xmin), mma->xmin);
  k_fill<<<nb, 256, 0, mma->stream>>>(mma->n, double(xmax), mma->xmax);
  OTM_CHECK_LAUNCH("k_fill");
  count_launches(2);
  return OTM_OK;
}

otm_status otm_mma_set_bound(otm_mma* mma, const float* xmin_dev, const float* xmax_dev) {
  if (!mma || !xmin_dev || !xmax_dev) return OTM_ERR_INVALID_ARGUMENT;
  const int nb = int(std::min<size_t>(kMaxPartials, (mma->n + 255) / 256));
  k_cast_f2d<<<nb, 256, 0, mma->stream>>>(mma->n, xmin_dev, mma->xmin);
  k_cast_f2d<<<nb, 256, 0, mma->stream>>>(mma->n, xmax_dev, mma->xmax);
  OTM_CHECK_LAUNCH("k_cast_f2d");
  count_launches(2);
  return OTM_OK;
}

otm_status otm_mma_update(otm_mma* mma, int itn, float* x_dev, const float* dfdx_dev, const float* gval_host,
                          const float* const* dgdx_dev) {
  if (!mma || !x_dev || !dfdx_dev || !gval_host || !dgdx_dev) return OTM_ERR_INVALID_ARGUMENT;
  cudaStream_t s = mma->stream;
  const size_t n = mma->n;
  const int nb = int(std::min<size_t>(kMaxPartials, (n + 255) / 256));
  k_cast_f2d<<<nb, 256, 0, s>>>(n, x_dev, mma->xvar);
  k_cast_f2d<<<nb, 256, 0, s>>>(n, dfdx_dev, mma->df0dx);
  for (int i = 0; i < mma->m; i++) {
    if (!dgdx_dev[i]) return OTM_ERR_INVALID_ARGUMENT;
    k_cast_f2d<<<nb, 256, 0, s>>>(n, dgdx_dev[i], mma->dgdx + i * n);
  }
  OTM_CHECK_LAUNCH("k_cast_f2d");
  count_launches(2 + mma->m);
  std::vector<double> gval(mma->m);
  for (int i = 0; i < mma->m; i++) gval[i] = gval_host[i];
  // f0val = 1 and move = 1 (optimization/mmaOptimizer.cu:69-70)
  OTM_TRY(mmasub_run(s, mma->m, n, itn, mma->xvar, mma->xmin, mma->xmax, mma->xold1, mma->xold2, mma->df0dx,
                     gval.data(), mma->dgdx, n, mma->low, mma->upp, mma->a0, mma->a.data(), mma->c.data(),
                     mma->d.data(), 1.0, mma->w, nullptr));
  k_cast_d2f<<<nb, 256, 0, s>>>(n, mma->xvar, x_dev);
  OTM_CHECK_LAUNCH("k_cast_d2f");
  count_launches(1);
  return OTM_OK;
}

otm_status otm_mmasub_device(int m, int n, int itn, double* xvar, double* xmin, double* xmax, double* xold1,
                             double* xold2, double f0val, double* df0dx, double* gval, otm_pitched_ptr dgdx,
                             double* low, double* upp, double a0, double* a, double* c, double* d, double move,
                             void* stream) {
  (void)f0val;  // unused by the reference as well
  if (m < 1 || m > kMmaMaxM || n < 1 || !xvar || !xmin || !xmax || !xold1 || !xold2 || !df0dx || !gval ||
      !dgdx.ptr || !low || !upp || !a || !c || !d || dgdx.pitch % sizeof(double) != 0 ||
      dgdx.pitch < size_t(n) * sizeof(double))
    return OTM_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<double> hg(m), ha(m), hc(m), hd(m);
  OTM_CUDA(cudaMemcpyAsync(hg.data(), gval, m * sizeof(double), cudaMemcpyDeviceToHost, s));
  OTM_CUDA(cudaMemcpyAsync(ha.data(), a, m * sizeof(double), cudaMemcpyDeviceToHost, s));
  OTM_CUDA(cudaMemcpyAsync(hc.data(), c, m * sizeof(double), cudaMemcpyDeviceToHost, s));
  OTM_CUDA(cudaMemcpyAsync(hd.data(), d, m * sizeof(double), cudaMemcpyDeviceToHost, s));
  OTM_CUDA(cudaStreamSynchronize(s));
  MmaWork w;
  otm_status st = work_alloc(w, m, size_t(n), s, true);
  if (st == OTM_OK)
    st = mmasub_run(s, m, size_t(n), itn, xvar, xmin, xmax, xold1, xold2, df0dx, hg.data(), (const double*)dgdx.ptr,
                    dgdx.pitch / sizeof(double), low, upp, a0, ha.data(), hc.data(), hd.data(), move, w, nullptr);
  work_free(w, s, true);
  return st;
}

}  // extern "C"
