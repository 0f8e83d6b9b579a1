// otm_cluster.cuh -- the lower part of the V-cycle in one launch of one thread-block cluster.
//
// The levels with at most kClMaxNv unknowns, down to and including the coarsest direct solve,
// run in kCl CTAs of one cluster. Every level is split into slabs of z-planes, one slab per
// CTA; each CTA keeps u and f of its planes (and r and the 27-point stencils of every level
// but the first) in its own shared memory. Values on a neighbouring CTA's planes are read
// through distributed shared memory, and the phases (colour passes, residual, restriction,
// coarsest solve, prolongation) are separated by cluster barriers instead of kernel
// boundaries, so the whole lower cycle costs one launch. The first level's stencils and
// residual stay in global memory (L2-resident). The arithmetic and its order are those of the
// per-level kernels in otm_mg_kernels.cuh; the coarsest solve is u = Ainv (f - mean f) as in
// k_coarsest_solve.
#pragma once

#include <cooperative_groups.h>

#include <algorithm>

#include "otm_mg_kernels.cuh"

namespace otm {

constexpr int kCl = 8;             // CTAs per cluster (portable cluster size)
constexpr int kClThreads = 512;
constexpr int kClMaxLevels = 8;
constexpr int kClMaxNv = 32768;    // unknowns of the first level handled by the cluster (32^3)
constexpr int kClMaxTab = 2048;    // plane-ownership entries over all levels

struct ClLevel {
  Dims d;
  int cs;      // case stride in shared memory: (planes of the fullest slab) * nx * ny
  int u_off;   // float offsets in shared memory
  int f_off;
  int r_off;   // < 0: residual in rg (global, lexicographic, case-major)
  int st_off;  // < 0: stencils read from st (global, colour-blocked)
  int tab_off; // first plane-ownership entry of this level
  int zstart[kCl + 1];  // CTA c holds planes [zstart[c], zstart[c+1])
  const float* st;
  float* rg;
};

struct ClDesc {
  int nlev;  // levels in the cluster part; the last one is the coarsest
  int pre, post;
  int nc;          // unknowns of the coarsest level
  int gather_off;  // float offset of the coarsest right-hand-side gather buffer (3 nc floats)
  int tab_base;    // float offset of the plane-ownership table (ints)
  ClLevel lv[kClMaxLevels];
  const float* f_in;  // right-hand side of the first level (global, case-major)
  float* u_out;       // its correction (global)
  const double* Ainv;
};

// Plane z of the vector at `off` of level L, wherever it lives in the cluster (case 0; case c
// is at + c * L.cs). tab entries are (rank << 16) | local plane.
__device__ __forceinline__ const float* cl_plane(const ClLevel& L, const int* tab, float* const* rb, int off,
                                                 int z) {
  const int e = tab[L.tab_off + z];
  return rb[e >> 16] + off + (e & 0xffff) * (L.d.nx * L.d.ny);
}

// One Gauss-Seidel colour pass over this CTA's vertices of the colour (gs_coarse_body);
// kSmemSt: the level's stencils are in shared memory (local layout [o][cs]).
template <bool kSmemSt>
__device__ __forceinline__ void cl_gs_t(const ClLevel& L, float* sm, const int* tab, float* const* rb, int rank,
                                        int color) {
  const Dims d = L.d;
  const int nx = d.nx, ny = d.ny, hx = nx >> 1, hy = ny >> 1, plane = nx * ny;
  const int z0 = L.zstart[rank], z1 = L.zstart[rank + 1];
  const int zf = z0 + (((z0 & 1) != (color >> 2)) ? 1 : 0);  // first own plane of the colour's parity
  const int npl = zf < z1 ? (z1 - zf + 1) >> 1 : 0;
  const int n = npl * hx * hy;
  const int cs = L.cs;
  const size_t nv = d.nv();
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int i = t % hx, j = (t / hx) % hy, pk = t / (hx * hy);
    const int x = 2 * i + (color & 1), y = 2 * j + ((color >> 1) & 1), z = zf + 2 * pk;
    const int xm = wrapm(x - 1, nx), xp = wrapm(x + 1, nx);
    const int ym = wrapm(y - 1, ny) * nx, y0 = y * nx, yp = wrapm(y + 1, ny) * nx;
    const float* pu[3] = {cl_plane(L, tab, rb, L.u_off, wrapm(z - 1, d.nz)), sm + L.u_off + (z - z0) * plane,
                          cl_plane(L, tab, rb, L.u_off, wrapm(z + 1, d.nz))};
    const int lidx = (z - z0) * plane + y0 + x;
    const float* sp = kSmemSt ? sm + L.st_off + lidx : L.st + cb_index(d, x, y, z);
    const size_t sstride = kSmemSt ? size_t(cs) : nv;
    float acc[3];
#pragma unroll
    for (int c = 0; c < 3; c++) acc[c] = sm[L.f_off + c * cs + lidx];
#pragma unroll
    for (int o = 0; o < 27; o++) {
      if (o == 13) continue;
      const float s = kSmemSt ? sp[o * sstride] : __ldg(sp + o * sstride);
      const int xo = o % 3 == 0 ? xm : (o % 3 == 1 ? x : xp);
      const int yo = (o / 3) % 3 == 0 ? ym : ((o / 3) % 3 == 1 ? y0 : yp);
      const float* q = pu[o / 9] + yo + xo;
#pragma unroll
      for (int c = 0; c < 3; c++) acc[c] -= s * q[c * cs];
    }
    const float s13 = kSmemSt ? sp[13 * sstride] : __ldg(sp + 13 * sstride);
    const float inv = 1.0f / s13;
#pragma unroll
    for (int c = 0; c < 3; c++) sm[L.u_off + c * cs + lidx] = acc[c] * inv;
  }
}

__device__ __forceinline__ void cl_gs(const ClLevel& L, float* sm, const int* tab, float* const* rb, int rank,
                                      int color) {
  if (L.st_off >= 0)
    cl_gs_t<true>(L, sm, tab, rb, rank, color);
  else
    cl_gs_t<false>(L, sm, tab, rb, rank, color);
}

// r = f - A u on this CTA's vertices (resid_coarse_body).
template <bool kSmemSt>
__device__ __forceinline__ void cl_resid_t(const ClLevel& L, float* sm, const int* tab, float* const* rb,
                                           int rank) {
  const Dims d = L.d;
  const int nx = d.nx, ny = d.ny, plane = nx * ny;
  const int z0 = L.zstart[rank], z1 = L.zstart[rank + 1];
  const int n = (z1 - z0) * plane;
  const int cs = L.cs;
  const size_t nv = d.nv();
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int zl = t / plane, rem = t - zl * plane, y = rem / nx, x = rem - y * nx, z = z0 + zl;
    const int xm = wrapm(x - 1, nx), xp = wrapm(x + 1, nx);
    const int ym = wrapm(y - 1, ny) * nx, y0 = y * nx, yp = wrapm(y + 1, ny) * nx;
    const float* pu[3] = {cl_plane(L, tab, rb, L.u_off, wrapm(z - 1, d.nz)), sm + L.u_off + zl * plane,
                          cl_plane(L, tab, rb, L.u_off, wrapm(z + 1, d.nz))};
    const float* sp = kSmemSt ? sm + L.st_off + t : L.st + cb_index(d, x, y, z);
    const size_t sstride = kSmemSt ? size_t(cs) : nv;
    float acc[3];
#pragma unroll
    for (int c = 0; c < 3; c++) acc[c] = sm[L.f_off + c * cs + t];
#pragma unroll
    for (int o = 0; o < 27; o++) {
      const float s = kSmemSt ? sp[o * sstride] : __ldg(sp + o * sstride);
      const int xo = o % 3 == 0 ? xm : (o % 3 == 1 ? x : xp);
      const int yo = (o / 3) % 3 == 0 ? ym : ((o / 3) % 3 == 1 ? y0 : yp);
      const float* q = pu[o / 9] + yo + xo;
#pragma unroll
      for (int c = 0; c < 3; c++) acc[c] -= s * q[c * cs];
    }
    if (L.r_off >= 0) {
#pragma unroll
      for (int c = 0; c < 3; c++) sm[L.r_off + c * cs + t] = acc[c];
    } else {
      const size_t g = size_t(z) * plane + rem;
#pragma unroll
      for (int c = 0; c < 3; c++) L.rg[c * nv + g] = acc[c];
    }
  }
}

__device__ __forceinline__ void cl_resid(const ClLevel& L, float* sm, const int* tab, float* const* rb, int rank) {
  if (L.st_off >= 0)
    cl_resid_t<true>(L, sm, tab, rb, rank);
  else
    cl_resid_t<false>(L, sm, tab, rb, rank);
}

// f_C = P^T r_F on this CTA's coarse vertices, and u_C = 0 there (restrict_body).
__device__ __forceinline__ void cl_restrict(const ClLevel& F, const ClLevel& C, float* sm, const int* tab,
                                            float* const* rb, int rank) {
  const Dims df = F.d, dc = C.d;
  const int pc = dc.nx * dc.ny, pf = df.nx * df.ny;
  const int Z0 = C.zstart[rank], Z1 = C.zstart[rank + 1];
  const int n = (Z1 - Z0) * pc;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int Zl = t / pc, rem = t - Zl * pc, Y = rem / dc.nx, X = rem - Y * dc.nx, Z = Z0 + Zl;
    const int xs[3] = {wrapm(2 * X - 1, df.nx), 2 * X, wrapm(2 * X + 1, df.nx)};
    const int ys[3] = {wrapm(2 * Y - 1, df.ny), 2 * Y, wrapm(2 * Y + 1, df.ny)};
    const int zs[3] = {wrapm(2 * Z - 1, df.nz), 2 * Z, wrapm(2 * Z + 1, df.nz)};
    const float* pr[3];
    int cstride;
    if (F.r_off >= 0) {
      cstride = F.cs;
#pragma unroll
      for (int k = 0; k < 3; k++) pr[k] = cl_plane(F, tab, rb, F.r_off, zs[k]);
    } else {
      cstride = int(df.nv());
#pragma unroll
      for (int k = 0; k < 3; k++) pr[k] = F.rg + size_t(zs[k]) * pf;
    }
    float acc[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int o = 0; o < 27; o++) {
      const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = o / 9 - 1;
      const float w = (ox ? 0.5f : 1.f) * (oy ? 0.5f : 1.f) * (oz ? 0.5f : 1.f);
      const float* q = pr[oz + 1] + ys[oy + 1] * df.nx + xs[ox + 1];
      // a global residual was written by other CTAs of this launch: read it past L1
#pragma unroll
      for (int c = 0; c < 3; c++) acc[c] += w * (F.r_off >= 0 ? q[c * cstride] : __ldcg(q + c * cstride));
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      sm[C.f_off + c * C.cs + t] = acc[c];
      sm[C.u_off + c * C.cs + t] = 0.f;
    }
  }
}

// u_C = Ainv (f_C - mean f_C) on this CTA's coarsest vertices (k_coarsest_solve): every CTA
// gathers the whole right-hand side, then one warp per own vertex forms the row product.
__device__ __forceinline__ void cl_coarsest(const ClDesc& cd, float* sm, const int* tab, float* const* rb,
                                            int rank, double* cmean) {
  const ClLevel& C = cd.lv[cd.nlev - 1];
  const int n = cd.nc, pc = C.d.nx * C.d.ny;
  float* g = sm + cd.gather_off;
  for (int idx = threadIdx.x; idx < 3 * n; idx += blockDim.x) {
    const int c = idx / n, v = idx - c * n, z = v / pc;
    g[idx] = cl_plane(C, tab, rb, C.f_off, z)[c * C.cs + (v - z * pc)];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < 3) {
    double s = 0.0;
    for (int i = lane; i < n; i += 32) s += double(g[warp * n + i]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) cmean[warp] = s / n;
  }
  __syncthreads();
  const int z0 = C.zstart[rank], z1 = C.zstart[rank + 1];
  const int nown = (z1 - z0) * pc;
  const double m0 = cmean[0], m1 = cmean[1], m2 = cmean[2];
  for (int t = warp; t < nown; t += int(blockDim.x >> 5)) {
    const int i = z0 * pc + t;  // lexicographic coarsest index
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int j = lane; j < n; j += 32) {
      const double m = __ldg(cd.Ainv + size_t(i) * n + j);  // symmetric: row i == column i
      a0 += m * (double(g[j]) - m0);
      a1 += m * (double(g[n + j]) - m1);
      a2 += m * (double(g[2 * n + j]) - m2);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      a0 += __shfl_xor_sync(0xffffffffu, a0, off);
      a1 += __shfl_xor_sync(0xffffffffu, a1, off);
      a2 += __shfl_xor_sync(0xffffffffu, a2, off);
    }
    if (lane == 0) {
      sm[C.u_off + t] = float(a0);
      sm[C.u_off + C.cs + t] = float(a1);
      sm[C.u_off + 2 * C.cs + t] = float(a2);
    }
  }
}

// u_F += P u_C on this CTA's fine vertices (prolong_body).
__device__ __forceinline__ void cl_prolong(const ClLevel& F, const ClLevel& C, float* sm, const int* tab,
                                           float* const* rb, int rank) {
  const Dims df = F.d, dc = C.d;
  const int pf = df.nx * df.ny;
  const int z0 = F.zstart[rank], z1 = F.zstart[rank + 1];
  const int n = (z1 - z0) * pf;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int zl = t / pf, rem = t - zl * pf, y = rem / df.nx, x = rem - y * df.nx, z = z0 + zl;
    const int X0 = x >> 1, Y0 = y >> 1, Z0 = z >> 1;
    const int X1 = (x & 1) ? wrapm(X0 + 1, dc.nx) : X0;
    const int Y1 = (y & 1) ? wrapm(Y0 + 1, dc.ny) : Y0;
    const int Z1 = (z & 1) ? wrapm(Z0 + 1, dc.nz) : Z0;
    const float wx1 = (x & 1) ? 0.5f : 0.f, wy1 = (y & 1) ? 0.5f : 0.f, wz1 = (z & 1) ? 0.5f : 0.f;
    const float wx0 = 1.f - wx1, wy0 = 1.f - wy1, wz0 = 1.f - wz1;
    const float* p0 = cl_plane(C, tab, rb, C.u_off, Z0);
    const float* p1 = cl_plane(C, tab, rb, C.u_off, Z1);
    const int r0 = Y0 * dc.nx, r1 = Y1 * dc.nx;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float* u0 = p0 + c * C.cs;
      const float* u1 = p1 + c * C.cs;
      const float a = wz0 * (wy0 * (wx0 * u0[r0 + X0] + wx1 * u0[r0 + X1]) +
                             wy1 * (wx0 * u0[r1 + X0] + wx1 * u0[r1 + X1])) +
                      wz1 * (wy0 * (wx0 * u1[r0 + X0] + wx1 * u1[r0 + X1]) +
                             wy1 * (wx0 * u1[r1 + X0] + wx1 * u1[r1 + X1]));
      float* uf = sm + F.u_off + c * F.cs + t;
      *uf = *uf + a;
    }
  }
}

static __global__ void __cluster_dims__(kCl, 1, 1) __launch_bounds__(kClThreads)
    k_vcycle_cluster(ClDesc cdp, const SolveScalars* sc) {
  // every CTA reads the same flag (written by earlier kernels), so the whole cluster leaves
  // together before any distributed shared memory access
  if (sc && solve_done(sc)) return;
  extern __shared__ __align__(16) float sm[];
  __shared__ float* rb[kCl];
  __shared__ double cmean[3];
  // the descriptor is indexed by level at run time: a shared copy keeps it out of local memory
  __shared__ ClDesc cd;
  {
    const int* src = reinterpret_cast<const int*>(&cdp);
    int* dst = reinterpret_cast<int*>(&cd);
    for (int i = threadIdx.x; i < int(sizeof(ClDesc) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  cooperative_groups::cluster_group cluster = cooperative_groups::this_cluster();
  const int rank = int(cluster.block_rank());
  if (threadIdx.x < kCl) rb[threadIdx.x] = cluster.map_shared_rank(sm, int(threadIdx.x));
  int* tab = reinterpret_cast<int*>(sm + cd.tab_base);
  const int L = cd.nlev;
  for (int l = 0; l < L; l++) {
    const ClLevel& V = cd.lv[l];
    for (int z = threadIdx.x; z < V.d.nz; z += blockDim.x) {
      int c = 0;
      while (c < kCl - 1 && z >= V.zstart[c + 1]) c++;
      tab[V.tab_off + z] = (c << 16) | (z - V.zstart[c]);
    }
  }
  // own planes: right-hand side of the first level, zero correction; stencils of the others
  {
    const ClLevel& T = cd.lv[0];
    const int pl = T.d.nx * T.d.ny, z0 = T.zstart[rank];
    const int n = (T.zstart[rank + 1] - z0) * pl;
    const size_t nv = T.d.nv();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      const size_t g = size_t(z0) * pl + t;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        sm[T.f_off + c * T.cs + t] = __ldg(cd.f_in + c * nv + g);
        sm[T.u_off + c * T.cs + t] = 0.f;
      }
    }
  }
  for (int l = 1; l < L - 1; l++) {
    const ClLevel& V = cd.lv[l];
    const int nx = V.d.nx, pl = nx * V.d.ny, z0 = V.zstart[rank];
    const int n = (V.zstart[rank + 1] - z0) * pl;
    const size_t nv = V.d.nv();
    for (int idx = threadIdx.x; idx < 27 * n; idx += blockDim.x) {
      const int o = idx / n, t = idx - o * n;
      const int zl = t / pl, rem = t - zl * pl, y = rem / nx, x = rem - y * nx;
      sm[V.st_off + o * V.cs + t] = __ldg(V.st + size_t(o) * nv + cb_index(V.d, x, y, z0 + zl));
    }
  }
  cluster.sync();
  for (int l = 0; l < L - 1; l++) {
    const ClLevel& F = cd.lv[l];
    for (int s = 0; s < cd.pre; s++)
      for (int c = 0; c < 8; c++) {
        cl_gs(F, sm, tab, rb, rank, c);
        cluster.sync();
      }
    cl_resid(F, sm, tab, rb, rank);
    cluster.sync();
    cl_restrict(F, cd.lv[l + 1], sm, tab, rb, rank);
    cluster.sync();
  }
  cl_coarsest(cd, sm, tab, rb, rank, cmean);
  cluster.sync();
  for (int l = L - 2; l >= 0; l--) {
    const ClLevel& F = cd.lv[l];
    cl_prolong(F, cd.lv[l + 1], sm, tab, rb, rank);
    cluster.sync();
    for (int s = 0; s < cd.post; s++)
      for (int c = 7; c >= 0; c--) {
        cl_gs(F, sm, tab, rb, rank, c);
        cluster.sync();
      }
  }
  // no distributed access after the last barrier: write this CTA's planes of the correction
  {
    const ClLevel& T = cd.lv[0];
    const int pl = T.d.nx * T.d.ny, z0 = T.zstart[rank];
    const int n = (T.zstart[rank + 1] - z0) * pl;
    const size_t nv = T.d.nv();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      const size_t g = size_t(z0) * pl + t;
#pragma unroll
      for (int c = 0; c < 3; c++) cd.u_out[c * nv + g] = sm[T.u_off + c * T.cs + t];
    }
  }
}

// Host-side layout of the cluster part for the level dimensions dims[0..n-1] (the last one is
// the coarsest). Returns the dynamic shared memory in bytes, or 0 when the levels do not fit
// one cluster (then the per-level kernels are used).
inline size_t cl_plan(const Dims* dims, int n, ClDesc* cd) {
  if (n < 2 || n > kClMaxLevels) return 0;
  if (dims[0].nv() > size_t(kClMaxNv)) return 0;
  int off = 0, tab = 0;
  for (int l = 0; l < n; l++) {
    const Dims d = dims[l];
    ClLevel& V = cd->lv[l];
    V = ClLevel{};
    V.d = d;
    if (l < n - 1 && ((d.nx | d.ny | d.nz) & 1)) return 0;  // smoothed levels are colour-split
    if (d.nz > 0xffff) return 0;
    int maxpl = 0;
    for (int c = 0; c <= kCl; c++) V.zstart[c] = int((long long)c * d.nz / kCl);
    for (int c = 0; c < kCl; c++) maxpl = std::max(maxpl, V.zstart[c + 1] - V.zstart[c]);
    V.cs = maxpl * d.nx * d.ny;
    V.u_off = off;
    off += 3 * V.cs;
    V.f_off = off;
    off += 3 * V.cs;
    V.r_off = -1;
    V.st_off = -1;
    if (l > 0 && l < n - 1) {
      V.r_off = off;
      off += 3 * V.cs;
      V.st_off = off;
      off += 27 * V.cs;
    }
    V.tab_off = tab;
    tab += d.nz;
  }
  cd->nlev = n;
  cd->nc = int(dims[n - 1].nv());
  cd->gather_off = off;
  off += 3 * cd->nc;
  cd->tab_base = off;
  off += tab;
  if (tab > kClMaxTab) return 0;
  const size_t bytes = size_t(off) * sizeof(float);
  if (bytes > size_t(kMaxDynSmem)) return 0;
  return bytes;
}

}  // namespace otm
