// otm_cluster.cuh -- the lower part of the V-cycle in one launch of one thread-block cluster.
//
// The levels with at most kClMaxNv unknowns, down to and including the coarsest direct solve,
// run in kCl CTAs of one cluster. Every level is split into slabs of z-planes, one slab per
// CTA; each CTA keeps u of its planes plus ghost copies of the two neighbouring planes, and f,
// r and the 27-point stencils of its planes (a first level too large for that keeps its stencils,
// right-hand side and residual in global memory, L2-resident), in its own shared memory. A CTA that writes
// an edge plane of u also stores the values into its neighbours' ghost copies (distributed
// shared memory), so colour passes and residuals read only local shared memory; restriction,
// prolongation and the coarsest gather read other CTAs' planes directly. The phases are
// separated by cluster barriers (barrier.cluster arrive/wait, release/acquire) instead of
// kernel boundaries, so the whole lower cycle costs one launch. A cluster barrier costs about
// as much as a small level's colour pass, so a sweep takes two: colours 0-3 update only the
// even planes and colours 4-7 only the odd ones, and within each half a vertex's changing
// neighbours lie in its own plane, held by its own CTA (CTA barriers between those passes). The arithmetic is that of the
// per-level kernels in otm_mg_kernels.cuh except for the summation order of the 27-point
// products; the coarsest solve is u = Ainv (f - mean f) as in k_coarsest_solve.
#pragma once

#include <cooperative_groups.h>

#include <algorithm>
#include <vector>

#include "otm_mg_kernels.cuh"

namespace otm {

constexpr int kCl = 16;            // CTAs per cluster (non-portable size, opted in at set-up): one
                                   // 32^3 colour pass at 16 CTAs loads half the stencils per SM of 8
constexpr int kClThreads = 512;
constexpr int kClMaxLevels = 8;
constexpr int kClMaxNv = 32768;    // unknowns of the first level handled by the cluster (32^3)
constexpr int kClMaxTab = 6144;    // plane-table entries over all levels (3 per plane)

struct ClLevel {
  Dims d;
  int cs;      // case stride of f and r in shared memory: (planes of the fullest slab) * nx * ny
  int urs;     // u row stride (nx, padded against shared-memory bank conflicts)
  int ups;     // u plane stride (ny * urs, padded)
  int ucs;     // u case stride: two more planes (ghost copies of the neighbouring slabs' edge planes)
  int u_off;   // float offsets in shared memory
  int f_off;   // < 0: right-hand side read from f_in (global; first level only, when not staged)
  int r_off;   // < 0: residual in rg (global, lexicographic, case-major)
  int st_off;  // < 0: stencils read from st (global, colour-blocked); else [vertex][27]
  int inv_off; // inverse diagonal per own vertex (with st_off >= 0)
  int tab_off; // plane tables of this level: nz ownership entries, then 2 nz ghost-push entries
  int tw_res;  // log2 of the lanes that share one vertex's 27 products in the residual
  int lhx, lhy;  // log2 of nx/2, ny/2 rounded up to powers of two (colour-pass enumeration)
  int lnx, lny;  // log2 of nx, ny rounded up (residual enumeration)
  int zstart[kCl + 1];  // CTA c holds planes [zstart[c], zstart[c+1])
  const float* st;
  float* rg;
};

struct ClDesc {
  int nlev;  // levels in the cluster part; the last one is the coarsest
  int pre, post;
  int nc;          // unknowns of the coarsest level
  int gather_off;  // float offset of the coarsest right-hand-side gather buffer (3 nc floats)
  int tab_base;    // float offset of the plane tables (ints)
  int ntab;        // their entries (cl_tables), copied from tab_g at the start of a call
  const int* tab_g;
  ClLevel lv[kClMaxLevels];
  const float* f_in;  // right-hand side of the first level (global, case-major)
  float* u_out;       // its correction (global)
  const double* Ainv;
};

// Layout of u on a CTA that holds planes [z0, z1): local plane 0 is a copy of plane z0 - 1,
// planes 1..z1-z0 are its own, plane z1-z0+1 a copy of plane z1 (periodic). A CTA that writes
// an edge plane also writes the value into the copies held by its neighbours ("ghost push"),
// so every read of a colour pass or residual is a local shared-memory load.

// Plane z of f or r (in-plane stride nx) at `off` of level L, wherever it lives in the cluster
// (case 0; case c is at + c * L.cs).
__device__ __forceinline__ const float* cl_plane(const ClLevel& L, const int* tab, float* const* rb, int off, int z) {
  const int e = tab[L.tab_off + z];
  return rb[e >> 16] + off + (e & 0xffff) * (L.d.nx * L.d.ny);
}

// Plane z of u (row stride urs; own planes start at local plane 1; case c at + c * L.ucs).
__device__ __forceinline__ const float* cl_uplane(const ClLevel& L, const int* tab, float* const* rb, int z) {
  const int e = tab[L.tab_off + z];
  return rb[e >> 16] + L.u_off + ((e & 0xffff) + 1) * L.ups;
}

// The ghost copies of plane z of u held by the neighbouring CTAs, at in-plane u index p of case
// 0 (null where plane z feeds fewer than two ghost copies). Taken before the stores of a vertex.
__device__ __forceinline__ void cl_ghosts(const ClLevel& L, const int* tab, float* const* rb, int z, int p,
                                          float*& g0, float*& g1) {
  const int* pt = tab + L.tab_off + L.d.nz + 2 * z;
  const int e0 = pt[0], e1 = pt[1];
  g0 = e0 >= 0 ? rb[e0 >> 16] + L.u_off + (e0 & 0xffff) * L.ups + p : nullptr;
  g1 = e1 >= 0 ? rb[e1 >> 16] + L.u_off + (e1 & 0xffff) * L.ups + p : nullptr;
}

// 27-point products of one vertex shared by a team of kTw lanes of one warp: lane k of the
// team takes the offsets k, k + kTw, ... and the team sums with butterfly shuffles, so small
// levels (a few dozen vertices per CTA) keep the latency of one vertex short. pu[0..2] are the
// local u planes z-1, z, z+1. Returns sum_o A(v, v+o) u(v+o) over the selected offsets in
// every lane of the team.
template <bool kSmemSt, bool kSkipCentre, int kTw>
__device__ __forceinline__ void cl_apply_team(const float* sp, size_t sstride, const float* const (&pu)[3], int xm,
                                              int x, int xp, int ym, int y0, int yp, int ucs, int lane,
                                              float (&acc)[3]) {
  acc[0] = acc[1] = acc[2] = 0.f;
  // fully unrolled (predicated) so that all loads of a lane are in flight together
#pragma unroll
  for (int k = 0; k < (27 + kTw - 1) / kTw; k++) {
    const int o = lane + k * kTw;
    if (o < 27 && !(kSkipCentre && o == 13)) {
      const float s = kSmemSt ? sp[o * sstride] : __ldg(sp + o * sstride);
      const int ox = o % 3, oy = (o / 3) % 3, oz = o / 9;
      const int xo = ox == 0 ? xm : (ox == 1 ? x : xp);
      const int yo = oy == 0 ? ym : (oy == 1 ? y0 : yp);
      const float* q = (oz == 0 ? pu[0] : (oz == 1 ? pu[1] : pu[2])) + yo + xo;
#pragma unroll
      for (int c = 0; c < 3; c++) acc[c] += s * q[c * ucs];
    }
  }
#pragma unroll
  for (int off = kTw >> 1; off > 0; off >>= 1)
#pragma unroll
    for (int c = 0; c < 3; c++) acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], off);
}

// One Gauss-Seidel colour pass over this CTA's vertices of the colour (gs_coarse_body); updated
// edge-plane values are pushed to the ghosts. Vertices are enumerated over power-of-two index
// ranges (shifts and masks instead of divisions); indices past nx/2 or ny/2 are idle. Only the
// warps that hold a vertex run the body, and every load of a vertex (right-hand side, inverse
// diagonal, ghost targets) is issued before its first store, so no store orders a reload.
template <bool kSmemSt, int kTwl>
__device__ __forceinline__ void cl_gs_t(const ClLevel& L, const float* __restrict__ f_glob, float* sm, const int* tab,
                                        float* const* rb, int rank, int color) {
  const Dims d = L.d;
  const int nx = d.nx, ny = d.ny, hx = nx >> 1, hy = ny >> 1, plane = nx * ny;
  const int z0 = L.zstart[rank], z1 = L.zstart[rank + 1];
  const int zf = z0 + (((z0 & 1) != (color >> 2)) ? 1 : 0);  // first own plane of the colour's parity
  const int npl = zf < z1 ? (z1 - zf + 1) >> 1 : 0;
  const int lhx = L.lhx, lhy = L.lhy;
  const int n = npl << (lhx + lhy);
  if (n == 0) return;  // uniform over the CTA
  const int cs = L.cs, ucs = L.ucs, urs = L.urs, ups = L.ups;
  const int u_off = L.u_off, f_off = L.f_off, st_off = L.st_off, inv_off = L.inv_off;
  const float* st_glob = L.st;
  const size_t nv = d.nv();
  // whole warps only (the team shuffles need all 32 lanes of a warp)
  const int total = ((n << kTwl) + 31) & ~31;
  for (int g = threadIdx.x; g < total; g += blockDim.x) {
    const int t0 = g >> kTwl, lane = g & ((1 << kTwl) - 1);
    const int i0 = t0 & ((1 << lhx) - 1), j0 = (t0 >> lhx) & ((1 << lhy) - 1), pk0 = t0 >> (lhx + lhy);
    const bool active = t0 < n && i0 < hx && j0 < hy;
    const int i = active ? i0 : 0, j = active ? j0 : 0, pk = active ? pk0 : 0;
    const int x = 2 * i + (color & 1), y = 2 * j + ((color >> 1) & 1), z = zf + 2 * pk;
    const int xm = wrapm(x - 1, nx), xp = wrapm(x + 1, nx);
    const int ym = wrapm(y - 1, ny) * urs, y0 = y * urs, yp = wrapm(y + 1, ny) * urs;
    const int zl = z - z0;
    const float* uz = sm + u_off + zl * ups;  // local planes zl, zl+1, zl+2 = z-1, z, z+1
    const float* const pu[3] = {uz, uz + ups, uz + 2 * ups};
    const int lidx = zl * plane + y * nx + x;  // own-vertex index (f, r, stencils)
    const float* sp = kSmemSt ? sm + st_off + lidx * 27 : st_glob + cb_index(d, x, y, z);
    const size_t sstride = kSmemSt ? size_t(1) : nv;
    float acc[3];
    cl_apply_team<kSmemSt, true, (1 << kTwl)>(sp, sstride, pu, xm, x, xp, ym, y0, yp, ucs, lane, acc);
    if (active && lane == 0) {
      const float inv = kSmemSt ? sm[inv_off + lidx] : 1.0f / __ldg(sp + 13 * sstride);
      float fv[3];
#pragma unroll
      for (int c = 0; c < 3; c++)
        fv[c] = f_off >= 0 ? sm[f_off + c * cs + lidx] : __ldg(f_glob + c * nv + size_t(z) * plane + y * nx + x);
      const int pu_idx = y0 + x;
      float *g0, *g1;
      cl_ghosts(L, tab, rb, z, pu_idx, g0, g1);
      float* own = sm + u_off + (zl + 1) * ups + pu_idx;
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float v = (fv[c] - acc[c]) * inv;
        own[c * ucs] = v;
        if (g0) g0[c * ucs] = v;
        if (g1) g1[c * ucs] = v;
      }
    }
  }
}

// One lane per vertex on every level: the 27 products with compile-time offsets cost fewer
// instructions than a lane team's shared offsets and shuffles, and on the small levels the
// pass is bound by instruction issue, not by the latency of one vertex.
__device__ __forceinline__ void cl_gs(const ClLevel& L, const float* f_glob, float* sm, const int* tab,
                                      float* const* rb, int rank, int color) {
  if (L.st_off < 0)
    cl_gs_t<false, 0>(L, f_glob, sm, tab, rb, rank, color);
  else
    cl_gs_t<true, 0>(L, f_glob, sm, tab, rb, rank, color);
}

// r = f - A u on this CTA's vertices (resid_coarse_body, the sum formed by a lane team).
template <bool kSmemSt, int kTwl>
__device__ __forceinline__ void cl_resid_t(const ClLevel& L, const float* __restrict__ f_glob, float* sm,
                                           int rank) {
  const Dims d = L.d;
  const int nx = d.nx, ny = d.ny, plane = nx * ny;
  const int z0 = L.zstart[rank], z1 = L.zstart[rank + 1];
  const int lnx = L.lnx, lny = L.lny;
  const int n = (z1 - z0) << (lnx + lny);
  if (n == 0) return;  // uniform over the CTA
  const int cs = L.cs, ucs = L.ucs, urs = L.urs, ups = L.ups;
  const int u_off = L.u_off, f_off = L.f_off, r_off = L.r_off, st_off = L.st_off;
  const float* st_glob = L.st;
  float* rg = L.rg;
  const size_t nv = d.nv();
  const int total = ((n << kTwl) + 31) & ~31;  // whole warps only
  for (int g = threadIdx.x; g < total; g += blockDim.x) {
    const int t0 = g >> kTwl, lane = g & ((1 << kTwl) - 1);
    const int x0 = t0 & ((1 << lnx) - 1), y0i = (t0 >> lnx) & ((1 << lny) - 1), zl0 = t0 >> (lnx + lny);
    const bool active = t0 < n && x0 < nx && y0i < ny;
    const int x = active ? x0 : 0, y = active ? y0i : 0, zl = active ? zl0 : 0;
    const int z = z0 + zl;
    const int xm = wrapm(x - 1, nx), xp = wrapm(x + 1, nx);
    const int ym = wrapm(y - 1, ny) * urs, y0 = y * urs, yp = wrapm(y + 1, ny) * urs;
    const float* uz = sm + u_off + zl * ups;
    const float* const pu[3] = {uz, uz + ups, uz + 2 * ups};
    const int lidx = zl * plane + y * nx + x;
    const float* sp = kSmemSt ? sm + st_off + lidx * 27 : st_glob + cb_index(d, x, y, z);
    const size_t sstride = kSmemSt ? size_t(1) : nv;
    float acc[3];
    cl_apply_team<kSmemSt, false, (1 << kTwl)>(sp, sstride, pu, xm, x, xp, ym, y0, yp, ucs, lane, acc);
    if (active && lane == 0) {
      const size_t gi = size_t(z) * plane + y * nx + x;
      float fv[3];  // all loads before the first store
#pragma unroll
      for (int c = 0; c < 3; c++) fv[c] = f_off >= 0 ? sm[f_off + c * cs + lidx] : __ldg(f_glob + c * nv + gi);
#pragma unroll
      for (int c = 0; c < 3; c++) {
        if (r_off >= 0)
          sm[r_off + c * cs + lidx] = fv[c] - acc[c];
        else
          rg[c * nv + gi] = fv[c] - acc[c];
      }
    }
  }
}

__device__ __forceinline__ void cl_resid(const ClLevel& L, const float* f_glob, float* sm, int rank) {
  if (L.st_off < 0)
    cl_resid_t<false, 0>(L, f_glob, sm, rank);
  else if (L.tw_res >= 3)
    cl_resid_t<true, 3>(L, f_glob, sm, rank);
  else
    cl_resid_t<true, 0>(L, f_glob, sm, rank);
}

// u = 0 on this CTA's planes of a level, ghost copies included.
__device__ __forceinline__ void cl_zero_u(const ClLevel& L, float* sm, int rank) {
  const int n = (L.zstart[rank + 1] - L.zstart[rank] + 2) * L.ups;
  for (int idx = threadIdx.x; idx < 3 * n; idx += blockDim.x) {
    const int c = idx / n;
    sm[L.u_off + c * L.ucs + (idx - c * n)] = 0.f;
  }
}

// f_C = P^T r_F on this CTA's coarse vertices (restrict_body).
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
    for (int c = 0; c < 3; c++) sm[C.f_off + c * C.cs + t] = acc[c];
  }
  cl_zero_u(C, sm, rank);
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
      const int zl = t / pc, rem = t - zl * pc, y = rem / C.d.nx, x = rem - y * C.d.nx;
      float* u = sm + C.u_off + (zl + 1) * C.ups + y * C.urs + x;  // own planes start at local plane 1
      u[0] = float(a0);
      u[C.ucs] = float(a1);
      u[2 * C.ucs] = float(a2);
    }
  }
}

// u_F += P u_C on this CTA's fine vertices (prolong_body); edge-plane results pushed to ghosts.
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
    const float* p0 = cl_uplane(C, tab, rb, Z0);
    const float* p1 = cl_uplane(C, tab, rb, Z1);
    const int r0 = Y0 * C.urs, r1 = Y1 * C.urs;
    const int pu_idx = y * F.urs + x;
    // every load (coarse values, possibly in other CTAs, the old fine values and the ghost
    // targets) before the first store
    float a[3], uo[3];
    float* uf = sm + F.u_off + (zl + 1) * F.ups + pu_idx;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float* u0 = p0 + c * C.ucs;
      const float* u1 = p1 + c * C.ucs;
      a[c] = wz0 * (wy0 * (wx0 * u0[r0 + X0] + wx1 * u0[r0 + X1]) +
                    wy1 * (wx0 * u0[r1 + X0] + wx1 * u0[r1 + X1])) +
             wz1 * (wy0 * (wx0 * u1[r0 + X0] + wx1 * u1[r0 + X1]) +
                    wy1 * (wx0 * u1[r1 + X0] + wx1 * u1[r1 + X1]));
      uo[c] = uf[c * F.ucs];
    }
    float *g0, *g1;
    cl_ghosts(F, tab, rb, z, pu_idx, g0, g1);
    const int fucs = F.ucs;
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const float v = uo[c] + a[c];
      uf[c * fucs] = v;
      if (g0) g0[c * fucs] = v;
      if (g1) g1[c * fucs] = v;
    }
  }
}

// One colour pass (cl_gs) followed by the barrier that its successor in the sweep needs:
// colours 0-3 update the even planes, 4-7 the odd ones, and a pass's changing neighbours are in
// its own plane unless it ends a half (colour 3 or 4 last, going up or down), after which the
// neighbouring CTAs' planes must be visible.
template <typename Cluster>
__device__ __forceinline__ void cl_gs_sync(const ClLevel& L, const float* f_glob, float* sm, const int* tab,
                                           float* const* rb, int rank, int color, bool half_end, Cluster& cluster) {
  cl_gs(L, f_glob, sm, tab, rb, rank, color);
  if (half_end)
    cluster.sync();
  else
    __syncthreads();
}

static __global__ void __cluster_dims__(kCl, 1, 1) __launch_bounds__(kClThreads)
    k_vcycle_cluster(ClDesc cdp, const SolveScalars* sc) {
  pdl_wait();
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
  // other CTAs' shared memory through the cluster window, this CTA's own directly
  if (threadIdx.x < kCl) rb[threadIdx.x] = int(threadIdx.x) == rank ? sm : cluster.map_shared_rank(sm, int(threadIdx.x));
  int* tab = reinterpret_cast<int*>(sm + cd.tab_base);
  const int L = cd.nlev;
  // plane tables (built on the host by cl_tables): owner and local plane of every plane, and the
  // ghost copies every plane feeds
  for (int i = threadIdx.x; i < cd.ntab; i += blockDim.x) tab[i] = __ldg(cd.tab_g + i);
  // the coarsest inverse is read once, late in the cycle: bring it into L2 now
  l2_prefetch_share(cd.Ainv, size_t(cd.nc) * size_t(cd.nc) * sizeof(double));
  // first level: zero correction (ghosts included) and, where it is staged, its right-hand side;
  // stencils of the other smoothed levels. One thread per own vertex, all of its loads in flight
  // before its stores (a copy of one element per round trip made this a chain of L2 latencies).
  cl_zero_u(cd.lv[0], sm, rank);
  if (cd.lv[0].f_off >= 0) {
    const ClLevel& V = cd.lv[0];
    const int pl = V.d.nx * V.d.ny, z0 = V.zstart[rank];
    const int n = (V.zstart[rank + 1] - z0) * pl;
    const size_t nv = V.d.nv();
    const float* fz = cd.f_in + size_t(z0) * pl;
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      float v[3];
#pragma unroll
      for (int c = 0; c < 3; c++) v[c] = __ldg(fz + c * nv + t);
#pragma unroll
      for (int c = 0; c < 3; c++) sm[V.f_off + c * V.cs + t] = v[c];
    }
  }
  for (int l = 0; l < L - 1; l++) {
    const ClLevel& V = cd.lv[l];
    if (V.st_off < 0) continue;
    const int nx = V.d.nx, pl = nx * V.d.ny, z0 = V.zstart[rank];
    const int n = (V.zstart[rank + 1] - z0) * pl;
    const size_t nv = V.d.nv();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      const int zl = t / pl, rem = t - zl * pl, y = rem / nx, x = rem - y * nx;
      const float* src = V.st + cb_index(V.d, x, y, z0 + zl);
      float a[27];
#pragma unroll
      for (int o = 0; o < 27; o++) a[o] = __ldg(src + size_t(o) * nv);
      float* dst = sm + V.st_off + t * 27;
#pragma unroll
      for (int o = 0; o < 27; o++) dst[o] = a[o];
      sm[V.inv_off + t] = 1.0f / a[13];
    }
  }
  cluster.sync();
  for (int l = 0; l < L - 1; l++) {
    const ClLevel& F = cd.lv[l];
    for (int s = 0; s < cd.pre; s++)
      for (int c = 0; c < 8; c++) cl_gs_sync(F, cd.f_in, sm, tab, rb, rank, c, c == 3 || c == 7, cluster);
    cl_resid(F, cd.f_in, sm, rank);
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
      for (int c = 7; c >= 0; c--) cl_gs_sync(F, cd.f_in, sm, tab, rb, rank, c, c == 4 || c == 0, cluster);
  }
  // no distributed access after the last barrier: write this CTA's planes of the correction
  {
    const ClLevel& T = cd.lv[0];
    const int pl = T.d.nx * T.d.ny, z0 = T.zstart[rank];
    const int n = (T.zstart[rank + 1] - z0) * pl;
    const size_t nv = T.d.nv();
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      const size_t g = size_t(z0) * pl + t;
      const int zl = t / pl, rem = t - zl * pl, y = rem / T.d.nx, x = rem - y * T.d.nx;
#pragma unroll
      for (int c = 0; c < 3; c++) cd.u_out[c * nv + g] = sm[T.u_off + c * T.ucs + (zl + 1) * T.ups + y * T.urs + x];
    }
  }
}

// Host-side layout of the cluster part for the level dimensions dims[0..n-1] (the last one is
// the coarsest). Returns the dynamic shared memory in bytes, or 0 when the levels do not fit
// one cluster (then the per-level kernels are used).
// Worst number of distinct shared-memory words per bank over the lane-team reads of u (teams of
// 8 lanes at vertices x, x+2, x+4, x+6; lane k reads offset k + 8 round) for row stride rs
// and plane stride ps.
inline int cl_team_conflicts(int rs, int ps) {
  int worst = 1;
  for (int round = 0; round < 4; round++) {
    int addr[32], na = 0;
    for (int j = 0; j < 4; j++)
      for (int lane = 0; lane < 8; lane++) {
        const int o = lane + 8 * round;
        if (o >= 27) continue;
        const int a = 2 * j + (o / 9) * ps + ((o / 3) % 3) * rs + o % 3;
        bool dup = false;
        for (int q = 0; q < na; q++) dup = dup || addr[q] == a;
        if (!dup) addr[na++] = a;
      }
    for (int b = 0; b < 32; b++) {
      int cnt = 0;
      for (int q = 0; q < na; q++) cnt += (addr[q] % 32) == b;
      worst = std::max(worst, cnt);
    }
  }
  return worst;
}

inline int cl_log2_ceil(int v) {
  int l = 0;
  while ((1 << l) < v) l++;
  return l;
}

// first_smem: the first level's stencils, right-hand side and residual also live in shared memory.
inline size_t cl_plan_try(const Dims* dims, int n, ClDesc* cd, bool first_smem) {
  if (n < 2 || n > kClMaxLevels) return 0;
  if (dims[0].nv() > size_t(kClMaxNv)) return 0;
  int off = 0, tab = 0;
  for (int l = 0; l < n; l++) {
    const Dims d = dims[l];
    ClLevel& V = cd->lv[l];
    V = ClLevel{};
    V.d = d;
    if (l < n - 1 && ((d.nx | d.ny | d.nz) & 1)) return 0;  // smoothed levels are colour-split
    if (d.nz > 0x7fff) return 0;
    int maxpl = 0;
    for (int c = 0; c <= kCl; c++) V.zstart[c] = int((long long)c * d.nz / kCl);
    for (int c = 0; c < kCl; c++) maxpl = std::max(maxpl, V.zstart[c + 1] - V.zstart[c]);
    const int plane = d.nx * d.ny;
    V.cs = maxpl * plane;
    // u strides: padded on the lane-team levels so that a round of team reads is free of bank
    // conflicts (smallest plane stride among the best), plain on the first level
    const bool smem_st = l < n - 1 && (l > 0 || first_smem);
    V.urs = d.nx;
    V.ups = plane;
    if (smem_st) {
      int best = cl_team_conflicts(V.urs, V.ups);
      for (int px = 0; px <= 32 && best > 1; px++)
        for (int py = 0; py < 64; py++) {
          const int rs = d.nx + px, ps = rs * d.ny + py;
          const int w = cl_team_conflicts(rs, ps);
          if (w < best || (w == best && ps < V.ups)) {
            best = w;
            V.urs = rs;
            V.ups = ps;
          }
        }
    }
    V.ucs = (maxpl + 2) * V.ups;
    V.u_off = off;
    off += 3 * V.ucs;
    V.f_off = -1;  // the first level reads its right-hand side from global memory unless staged
    if (l > 0 || smem_st) {
      V.f_off = off;
      off += 3 * V.cs;
    }
    V.r_off = V.st_off = V.inv_off = -1;
    if (smem_st) {
      V.r_off = off;
      off += 3 * V.cs;
      V.st_off = off;
      off += 27 * V.cs;
      V.inv_off = off;
      off += V.cs;
    }
    V.tab_off = tab;
    tab += 3 * d.nz;
    V.lhx = cl_log2_ceil(std::max(1, d.nx / 2));
    V.lhy = cl_log2_ceil(std::max(1, d.ny / 2));
    V.lnx = cl_log2_ceil(d.nx);
    V.lny = cl_log2_ceil(d.ny);
    // residual: 8 lanes per vertex where that fills about one round of the CTA's threads
    V.tw_res = (((maxpl << (V.lnx + V.lny)) << 3) <= 2 * kClThreads) ? 3 : 0;
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

// The plane tables of a plan, cd->ntab ints: per level (at tab_off) the owner CTA and local plane
// of every plane ((c << 16) | local), then for every plane the two ghost copies it feeds ((CTA <<
// 16) | local ghost plane, -1 for none): plane z is the lower ghost (local plane 0) of the CTA
// whose slab starts at z + 1 and the upper ghost (local plane slab + 1) of the CTA whose slab ends
// at z, periodically. Built once per plan on the host, copied into shared memory by every call.
inline void cl_tables(ClDesc* cd, std::vector<int>& tab) {
  int n = 0;
  for (int l = 0; l < cd->nlev; l++) n = std::max(n, cd->lv[l].tab_off + 3 * cd->lv[l].d.nz);
  tab.assign(size_t(n), 0);
  for (int l = 0; l < cd->nlev; l++) {
    const ClLevel& V = cd->lv[l];
    const int nz = V.d.nz;
    for (int z = 0; z < nz; z++) {
      int c = 0;
      while (c < kCl - 1 && z >= V.zstart[c + 1]) c++;
      tab[size_t(V.tab_off + z)] = (c << 16) | (z - V.zstart[c]);
      int k = 0;
      int* push = tab.data() + V.tab_off + nz + 2 * z;
      push[0] = push[1] = -1;
      for (int q = 0; q < kCl && k < 2; q++) {
        const int a = V.zstart[q], b = V.zstart[q + 1];
        if (b == a) continue;
        if ((a - 1 + nz) % nz == z) push[k++] = (q << 16) | 0;           // q's lower ghost
        if (k < 2 && b % nz == z) push[k++] = (q << 16) | (b - a + 1);   // q's upper ghost
      }
    }
  }
  cd->ntab = n;
}

// Host-side layout of the cluster part (see cl_plan_try): the first level's stencils in shared
// memory when everything fits, else in global memory.
inline size_t cl_plan(const Dims* dims, int n, ClDesc* cd) {
  const size_t b = cl_plan_try(dims, n, cd, true);
  return b ? b : cl_plan_try(dims, n, cd, false);
}

}  // namespace otm
