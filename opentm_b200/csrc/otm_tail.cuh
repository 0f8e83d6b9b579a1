// otm_tail.cuh -- the small end of the V-cycle in one launch.
//
// Every level with at most kTailMaxNv unknowns, down to and including the coarsest direct
// solve, runs inside a single 1024-thread CTA: the vectors u, f, r of those levels (3 load
// cases) live in shared memory, only the 27-point stencils and the coarsest inverse are read
// from global memory (L2-resident), and the phases (colour passes, residual, restriction,
// coarsest solve, prolongation) are separated by __syncthreads() instead of kernel
// boundaries. Same arithmetic and order as the per-level kernels of otm_mg_kernels.cuh.
#pragma once

#include "otm_mg_kernels.cuh"

namespace otm {

constexpr int kTailMaxNv = 4096;   // 16^3
constexpr int kTailMaxLevels = 8;
constexpr int kTailThreads = 1024;

struct TailLevel {
  Dims d;
  const float* st;  // colour-blocked for smoothed levels, lexicographic for the coarsest
  int off;          // float offset of this level's u in shared memory (f = u + 3nv, r = f + 3nv)
};

struct TailDesc {
  int nlev;  // levels in the tail (the last one is the coarsest)
  int pre, post;
  int nc;    // unknowns of the coarsest level
  TailLevel lv[kTailMaxLevels];
  const float* f_in;  // right-hand side of the first tail level (global, 3 cases)
  float* u_out;       // its correction (global)
  const double* Ainv;
};

__device__ __forceinline__ void tail_gs(const TailLevel& L, float* sm, int color) {
  const Dims d = L.d;
  const int hx = d.nx >> 1, hy = d.ny >> 1;
  const int nsub = int(d.nv() >> 3), nv = int(d.nv());
  float* u = sm + L.off;
  const float* f = u + 3 * nv;
  for (int t = threadIdx.x; t < nsub; t += blockDim.x) {
    const int i = t % hx, j = (t / hx) % hy, kq = t / (hx * hy);
    const int x = 2 * i + (color & 1), y = 2 * j + ((color >> 1) & 1), z = 2 * kq + (color >> 2);
    Nbr nb;
    nb.init(d, x, y, z);
    const int v = int(nb.at(13));
    const size_t sb = size_t(color) * nsub + t;
    float acc[3] = {f[v], f[nv + v], f[2 * nv + v]};
#pragma unroll
    for (int o = 0; o < 27; o++) {
      if (o == 13) continue;
      const float s = __ldg(L.st + size_t(o) * nv + sb);
      const int jn = int(nb.at(o));
      acc[0] -= s * u[jn];
      acc[1] -= s * u[nv + jn];
      acc[2] -= s * u[2 * nv + jn];
    }
    const float inv = 1.0f / __ldg(L.st + size_t(13) * nv + sb);
    u[v] = acc[0] * inv;
    u[nv + v] = acc[1] * inv;
    u[2 * nv + v] = acc[2] * inv;
  }
}

__device__ __forceinline__ void tail_resid(const TailLevel& L, float* sm) {
  const Dims d = L.d;
  const int nv = int(d.nv());
  const float* u = sm + L.off;
  const float* f = u + 3 * nv;
  float* r = sm + L.off + 6 * nv;
  for (int v = threadIdx.x; v < nv; v += blockDim.x) {
    const int x = v % d.nx, y = (v / d.nx) % d.ny, z = v / (d.nx * d.ny);
    Nbr nb;
    nb.init(d, x, y, z);
    const size_t sb = cb_index(d, x, y, z);
    float acc[3] = {f[v], f[nv + v], f[2 * nv + v]};
#pragma unroll
    for (int o = 0; o < 27; o++) {
      const float s = __ldg(L.st + size_t(o) * nv + sb);
      const int jn = int(nb.at(o));
      acc[0] -= s * u[jn];
      acc[1] -= s * u[nv + jn];
      acc[2] -= s * u[2 * nv + jn];
    }
    r[v] = acc[0];
    r[nv + v] = acc[1];
    r[2 * nv + v] = acc[2];
  }
}

__device__ __forceinline__ void tail_restrict(const TailLevel& F, const TailLevel& C, float* sm) {
  const int nvf = int(F.d.nv()), nvc = int(C.d.nv());
  const float* r = sm + F.off + 6 * nvf;
  float* fc = sm + C.off + 3 * nvc;
  for (int V = threadIdx.x; V < nvc; V += blockDim.x) {
    const int X = V % C.d.nx, Y = (V / C.d.nx) % C.d.ny, Z = V / (C.d.nx * C.d.ny);
    Nbr nb;
    nb.init(F.d, 2 * X, 2 * Y, 2 * Z);
    float acc[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int o = 0; o < 27; o++) {
      const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = o / 9 - 1;
      const float w = (ox ? 0.5f : 1.f) * (oy ? 0.5f : 1.f) * (oz ? 0.5f : 1.f);
      const int j = int(nb.at(o));
      acc[0] += w * r[j];
      acc[1] += w * r[nvf + j];
      acc[2] += w * r[2 * nvf + j];
    }
    fc[V] = acc[0];
    fc[nvc + V] = acc[1];
    fc[2 * nvc + V] = acc[2];
  }
}

__device__ __forceinline__ void tail_prolong(const TailLevel& F, const TailLevel& C, float* sm) {
  const int nvf = int(F.d.nv()), nvc = int(C.d.nv());
  float* uf = sm + F.off;
  const float* uc = sm + C.off;
  const Dims df = F.d, dc = C.d;
  for (int v = threadIdx.x; v < nvf; v += blockDim.x) {
    const int x = v % df.nx, y = (v / df.nx) % df.ny, z = v / (df.nx * df.ny);
    const int X0 = x >> 1, Y0 = y >> 1, Z0 = z >> 1;
    const int X1 = (x & 1) ? wrapm(X0 + 1, dc.nx) : X0;
    const int Y1 = (y & 1) ? wrapm(Y0 + 1, dc.ny) : Y0;
    const int Z1 = (z & 1) ? wrapm(Z0 + 1, dc.nz) : Z0;
    const float wx1 = (x & 1) ? 0.5f : 0.f, wy1 = (y & 1) ? 0.5f : 0.f, wz1 = (z & 1) ? 0.5f : 0.f;
    const float wx0 = 1.f - wx1, wy0 = 1.f - wy1, wz0 = 1.f - wz1;
    const int r00 = (Y0 + dc.ny * Z0) * dc.nx, r10 = (Y1 + dc.ny * Z0) * dc.nx;
    const int r01 = (Y0 + dc.ny * Z1) * dc.nx, r11 = (Y1 + dc.ny * Z1) * dc.nx;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float* u = uc + c * nvc;
      const float a = wz0 * (wy0 * (wx0 * u[r00 + X0] + wx1 * u[r00 + X1]) +
                             wy1 * (wx0 * u[r10 + X0] + wx1 * u[r10 + X1])) +
                      wz1 * (wy0 * (wx0 * u[r01 + X0] + wx1 * u[r01 + X1]) +
                             wy1 * (wx0 * u[r11 + X0] + wx1 * u[r11 + X1]));
      uf[c * nvf + v] += a;
    }
  }
}

// Coarsest level: u = Ainv (f - mean f), Ainv symmetric (column reads are coalesced).
__device__ __forceinline__ void tail_coarsest(const TailLevel& L, float* sm, const double* __restrict__ Ainv, int n) {
  float* u = sm + L.off;
  const float* f = u + 3 * n;
  __shared__ double mean[3];
  if (threadIdx.x < 3) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += f[threadIdx.x * n + i];
    mean[threadIdx.x] = s / n;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int j = 0; j < n; j++) {
      const double m = __ldg(Ainv + size_t(j) * n + i);
      a0 += m * (double(f[j]) - mean[0]);
      a1 += m * (double(f[n + j]) - mean[1]);
      a2 += m * (double(f[2 * n + j]) - mean[2]);
    }
    u[i] = float(a0);
    u[n + i] = float(a1);
    u[2 * n + i] = float(a2);
  }
}

__device__ __forceinline__ void vcycle_tail_body(const TailDesc& td, float* sm) {
  const int L = td.nlev;
  // load the first tail level's right-hand side
  {
    const int nv = int(td.lv[0].d.nv());
    float* f = sm + td.lv[0].off + 3 * nv;
    for (int i = threadIdx.x; i < 3 * nv; i += blockDim.x) f[i] = td.f_in[i];
  }
  __syncthreads();
  for (int l = 0; l < L - 1; l++) {
    const TailLevel& T = td.lv[l];
    const int nv = int(T.d.nv());
    float* u = sm + T.off;
    for (int i = threadIdx.x; i < 3 * nv; i += blockDim.x) u[i] = 0.f;
    __syncthreads();
    for (int s = 0; s < td.pre; s++)
      for (int c = 0; c < 8; c++) {
        tail_gs(T, sm, c);
        __syncthreads();
      }
    tail_resid(T, sm);
    __syncthreads();
    tail_restrict(T, td.lv[l + 1], sm);
    __syncthreads();
  }
  tail_coarsest(td.lv[L - 1], sm, td.Ainv, td.nc);
  __syncthreads();
  for (int l = L - 2; l >= 0; l--) {
    const TailLevel& T = td.lv[l];
    tail_prolong(T, td.lv[l + 1], sm);
    __syncthreads();
    for (int s = 0; s < td.post; s++)
      for (int c = 7; c >= 0; c--) {
        tail_gs(T, sm, c);
        __syncthreads();
      }
  }
  {
    const int nv = int(td.lv[0].d.nv());
    const float* u = sm + td.lv[0].off;
    for (int i = threadIdx.x; i < 3 * nv; i += blockDim.x) td.u_out[i] = u[i];
  }
}

static __global__ void __launch_bounds__(kTailThreads) k_vcycle_tail(TailDesc td, const SolveScalars* sc) {
  pdl_wait();
  if (sc && solve_done(sc)) return;
  extern __shared__ float sm[];
  vcycle_tail_body(td, sm);
}

}  // namespace otm
