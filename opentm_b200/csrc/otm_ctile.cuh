// otm_ctile.cuh -- tile-staged Gauss-Seidel sweeps of the coarse (27-point stencil) levels.
//
// The coarse levels' smoothing (homogenization/grid.cu:707-809, eight colours per sweep) runs one
// launch per sweep instead of one launch per colour: every CTA stages the correction u (3 cases)
// of a tile of 16 x 8 x 8 vertices plus a one-site halo in shared memory, runs the eight colour
// passes of the sweep inside the tile with the halo held at the values it had when the sweep
// started, and writes the interior to a second buffer. As on the fine level, consecutive sweeps
// alternate between two tilings shifted by half a tile along every axis, so that the faces of one
// tiling lie inside the tiles of the other, and the post-smoothing sweeps run in the reverse colour
// order on the mirrored tilings (the V-cycle stays symmetric for PCG). The first sweep after the
// coarse-grid correction adds the trilinear prolongation of the next coarser level's correction
// while it stages the tile.
//
// One thread per vertex of the current colour (8 x 4 x 4 per tile): it reads the 27 stencil
// coefficients of its vertex from the level's colour-blocked stencil array in global memory (lanes
// of a warp read consecutive entries), the 26 neighbours from shared memory, and the right-hand side
// from global memory. The staged sites are float4 {u_case0, u_case1, u_case2, 0} with the even and
// the odd sites of a row stored apart and rows padded to 19 entries, so that the lanes of a warp,
// which update every other site of a row, read consecutive entries.
#pragma once

#include "otm_tile.cuh"

namespace otm {

constexpr int kCTX = 16, kCTY = 8, kCTZ = 8;                      // interior vertices of a coarse tile
constexpr int kCSX = kCTX + 2, kCSY = kCTY + 2, kCSZ = kCTZ + 2;  // staged sites
constexpr int kCSHalf = kCSX / 2;
constexpr int kCSRow = kCSX + 1;                                  // padded row pitch (float4)
constexpr int kCSPlane = kCSRow * kCSY;                           // 190
constexpr int kCSSites = kCSPlane * kCSZ;                         // 1900
constexpr int kCThreads = (kCTX / 2) * (kCTY / 2) * (kCTZ / 2);   // 128: one per vertex of a colour
constexpr int kCCX = kCTX / 2 + 2, kCCY = kCTY / 2 + 2, kCCZ = kCTZ / 2 + 2;  // coarser block (10 x 6 x 6)
constexpr int kCCSites = kCCX * kCCY * kCCZ;
constexpr size_t kCTileSmem = size_t(kCSSites) * sizeof(float4);                               // 30,400 B
constexpr size_t kCTileSmemProlong = kCTileSmem + size_t(kCCSites) * sizeof(float4);            // 36,160 B

// Whether a coarse level can be tiled.
__host__ __device__ inline bool ctile_fits(const Dims& d) {
  return d.nx % kCTX == 0 && d.ny % kCTY == 0 && d.nz % kCTZ == 0;
}
__host__ __device__ inline unsigned ctile_count(const Dims& d) {
  return unsigned(d.nx / kCTX) * unsigned(d.ny / kCTY) * unsigned(d.nz / kCTZ);
}

__device__ __forceinline__ int csite(int lx, int ly, int lz) {
  return lz * kCSPlane + ly * kCSRow + ((lx & 1) ? kCSHalf + (lx >> 1) : (lx >> 1));
}

// Origin of coarse tile b of tiling `shift` (unwrapped, as tile_origin).
__device__ __forceinline__ void ctile_origin(const Dims& d, unsigned b, int shift, int& x0, int& y0, int& z0) {
  const unsigned ntx = unsigned(d.nx / kCTX), nty = unsigned(d.ny / kCTY);
  const unsigned q = b / ntx;
  x0 = int(b - q * ntx) * kCTX + shift * (kCTX / 2);
  y0 = int(q % nty) * kCTY + shift * (kCTY / 2);
  z0 = int(q / nty) * kCTZ + shift * (kCTZ / 2);
}

// Trilinear prolongation at the fine site (ux, uy, uz) (unwrapped) from the staged coarser block
// (float4 per site, origin c0); the expression and weights of prolong_body.
__device__ __forceinline__ float3 cprolong_site(const float4* cb, int ux, int uy, int uz, int c0x, int c0y, int c0z) {
  const int ax0 = (ux >> 1) - c0x, ay0 = (uy >> 1) - c0y, az0 = (uz >> 1) - c0z;
  const int ax1 = ax0 + (ux & 1), ay1 = ay0 + (uy & 1), az1 = az0 + (uz & 1);
  const float wx1 = (ux & 1) ? 0.5f : 0.f, wy1 = (uy & 1) ? 0.5f : 0.f, wz1 = (uz & 1) ? 0.5f : 0.f;
  const float wx0 = 1.f - wx1, wy0 = 1.f - wy1, wz0 = 1.f - wz1;
  const float4* r00 = cb + (ay0 + kCCY * az0) * kCCX;
  const float4* r10 = cb + (ay1 + kCCY * az0) * kCCX;
  const float4* r01 = cb + (ay0 + kCCY * az1) * kCCX;
  const float4* r11 = cb + (ay1 + kCCY * az1) * kCCX;
  const float4 a00 = r00[ax0], b00 = r00[ax1], a10 = r10[ax0], b10 = r10[ax1];
  const float4 a01 = r01[ax0], b01 = r01[ax1], a11 = r11[ax0], b11 = r11[ax1];
  float3 o;
  o.x = wz0 * (wy0 * (wx0 * a00.x + wx1 * b00.x) + wy1 * (wx0 * a10.x + wx1 * b10.x)) +
        wz1 * (wy0 * (wx0 * a01.x + wx1 * b01.x) + wy1 * (wx0 * a11.x + wx1 * b11.x));
  o.y = wz0 * (wy0 * (wx0 * a00.y + wx1 * b00.y) + wy1 * (wx0 * a10.y + wx1 * b10.y)) +
        wz1 * (wy0 * (wx0 * a01.y + wx1 * b01.y) + wy1 * (wx0 * a11.y + wx1 * b11.y));
  o.z = wz0 * (wy0 * (wx0 * a00.z + wx1 * b00.z) + wy1 * (wx0 * a10.z + wx1 * b10.z)) +
        wz1 * (wy0 * (wx0 * a01.z + wx1 * b01.z) + wy1 * (wx0 * a11.z + wx1 * b11.z));
  return o;
}

// One colour pass over the tile: the thread's vertex of colour (CX, CY, CZ).
// The operands of this thread's vertex in colour pass (CX, CY, CZ) that do not depend on u: its
// 27 stencil values and its right-hand side. They are fetched one pass ahead (while the previous
// pass computes), so the passes wait on shared memory only, not on L2.
struct CPassOps {
  float s[27];
  float f[3];
};

template <int CX, int CY, int CZ>
__device__ __forceinline__ void ctile_fetch(const Dims& d, int x0, int y0, int z0, const float* __restrict__ st,
                                            const float* __restrict__ f, CPassOps& ops) {
  const int t = int(threadIdx.x);
  const int i = t & 7, j = (t >> 3) & 3, k = t >> 5;
  const int lx = 1 + 2 * i + CX, ly = 1 + 2 * j + CY, lz = 1 + 2 * k + CZ;
  const int X = wrapm(x0 + lx - 1, d.nx), Y = wrapm(y0 + ly - 1, d.ny), Z = wrapm(z0 + lz - 1, d.nz);
  const size_t nv = d.nv();
  const size_t v = size_t(X) + size_t(d.nx) * (size_t(Y) + size_t(d.ny) * Z);
  const size_t sb = cb_index(d, X, Y, Z);
#pragma unroll
  for (int o = 0; o < 27; o++) ops.s[o] = __ldg(st + size_t(o) * nv + sb);
#pragma unroll
  for (int c = 0; c < 3; c++) ops.f[c] = __ldg(f + c * nv + v);
}

// One colour pass (CX, CY, CZ) of the tile's interior from fetched operands: each thread updates
// one vertex (128 threads: 8 x 4 x 4 vertices of the colour in the 16 x 8 x 8 tile).
template <int CX, int CY, int CZ>
__device__ __forceinline__ void ctile_apply(float4* sm, const CPassOps& ops) {
  const int t = int(threadIdx.x);
  const int i = t & 7, j = (t >> 3) & 3, k = t >> 5;
  const int lx = 1 + 2 * i + CX, ly = 1 + 2 * j + CY, lz = 1 + 2 * k + CZ;
  float acc[3] = {ops.f[0], ops.f[1], ops.f[2]};
  const float4* b = sm + csite(lx, ly, lz);
  // neighbour offsets: the parity of lx is fixed by the pass, so left / right are compile-time
  constexpr int oL = (CX == 0) ? -kCSHalf : kCSHalf - 1;  // lx odd for CX = 0
  constexpr int oR = (CX == 0) ? -kCSHalf + 1 : kCSHalf;
#pragma unroll
  for (int o = 0; o < 27; o++) {
    if (o == 13) continue;
    const int ox = o % 3 - 1, oy = (o / 3) % 3 - 1, oz = o / 9 - 1;
    const int off = (ox < 0 ? oL : (ox > 0 ? oR : 0)) + oy * kCSRow + oz * kCSPlane;
    const float4 n = b[off];
    acc[0] -= ops.s[o] * n.x;
    acc[1] -= ops.s[o] * n.y;
    acc[2] -= ops.s[o] * n.z;
  }
  const float inv = 1.0f / ops.s[13];
  sm[csite(lx, ly, lz)] = make_float4(acc[0] * inv, acc[1] * inv, acc[2] * inv, 0.f);
}

// Colour pass A from its fetched operands, with the operands of the next pass B fetched first.
// No barrier here: the caller separates the passes.
template <int AX, int AY, int AZ, int BX, int BY, int BZ>
__device__ __forceinline__ void ctile_step(float4* sm, const Dims& d, int x0, int y0, int z0,
                                           const float* __restrict__ st, const float* __restrict__ f,
                                           const CPassOps& cur, CPassOps& next) {
  ctile_fetch<BX, BY, BZ>(d, x0, y0, z0, st, f, next);
  ctile_apply<AX, AY, AZ>(sm, cur);
}

// One Gauss-Seidel sweep of a coarse level on the tiles of tiling `shift`: stage u from zero, from
// u_in, or from u_in plus the prolongation of the coarser correction uc (kStart as TileStart), run
// the eight colour passes in the order 0..7 (7..0 when `reverse`), write the interior to u_out
// (which must not alias u_in). st: the level's 27-point stencils (colour-blocked), f: its
// right-hand side, all FP32, 3 cases.
template <int kStart>
__global__ void __launch_bounds__(kCThreads)
    k_ctile_sweep(Dims d, Dims dc, const float* __restrict__ st, const float* __restrict__ u_in,
                  const float* __restrict__ uc, float* __restrict__ u_out, const float* __restrict__ f, int shift,
                  int reverse, const SolveScalars* sc) {
  extern __shared__ float4 csm[];
  float4* cb = csm + kCSSites;
  pdl_wait();
  if (sc && solve_done(sc)) return;
  int x0, y0, z0;
  ctile_origin(d, blockIdx.x, shift, x0, y0, z0);
  const size_t nv = d.nv();
  const int t = int(threadIdx.x);
  // the first pass's stencils and right-hand side, in flight during the staging
  CPassOps first;
  if (!reverse)
    ctile_fetch<0, 0, 0>(d, x0, y0, z0, st, f, first);
  else
    ctile_fetch<1, 1, 1>(d, x0, y0, z0, st, f, first);
  const int c0x = x0 / 2 - 1, c0y = y0 / 2 - 1, c0z = z0 / 2 - 1;
  // staging: every thread first issues all its global loads (the coarser block, then the sites of
  // the staged box in natural order), then stores
  constexpr int kSI = (kCSX * kCSY * kCSZ + kCThreads - 1) / kCThreads;
  constexpr int kCI = (kCCSites + kCThreads - 1) / kCThreads;
  float cbv[kStart == kFromUProlong ? kCI : 1][3];
  if (kStart == kFromUProlong) {
    const size_t nvc = dc.nv();
#pragma unroll
    for (int it = 0; it < kCI; it++) {
      const int q = t + it * kCThreads;
      if (q < kCCSites) {
        const int ax = q % kCCX, ay = (q / kCCX) % kCCY, az = q / (kCCX * kCCY);
        const int X = wrapm(c0x + ax, dc.nx), Y = wrapm(c0y + ay, dc.ny), Z = wrapm(c0z + az, dc.nz);
        const size_t g = size_t(X) + size_t(dc.nx) * (size_t(Y) + size_t(dc.ny) * Z);
#pragma unroll
        for (int c = 0; c < 3; c++) cbv[it][c] = __ldg(uc + c * nvc + g);
      }
    }
  }
  float uv[kStart != kFromZero ? kSI : 1][3];
  if (kStart != kFromZero) {
#pragma unroll
    for (int it = 0; it < kSI; it++) {
      const int q = t + it * kCThreads;
      if (q < kCSX * kCSY * kCSZ) {
        const int lx = q % kCSX, ly = (q / kCSX) % kCSY, lz = q / (kCSX * kCSY);
        const size_t g = size_t(wrapm(x0 - 1 + lx, d.nx)) +
                         size_t(d.nx) * (size_t(wrapm(y0 - 1 + ly, d.ny)) + size_t(d.ny) * wrapm(z0 - 1 + lz, d.nz));
#pragma unroll
        for (int c = 0; c < 3; c++) uv[it][c] = __ldg(u_in + c * nv + g);
      }
    }
  }
  if (kStart == kFromUProlong) {
#pragma unroll
    for (int it = 0; it < kCI; it++) {
      const int q = t + it * kCThreads;
      if (q < kCCSites) cb[q] = make_float4(cbv[it][0], cbv[it][1], cbv[it][2], 0.f);
    }
    __syncthreads();
  }
#pragma unroll
  for (int it = 0; it < kSI; it++) {
    const int q = t + it * kCThreads;
    if (q < kCSX * kCSY * kCSZ) {
      const int lx = q % kCSX, ly = (q / kCSX) % kCSY, lz = q / (kCSX * kCSY);
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (kStart != kFromZero) {
        v.x = uv[it][0];
        v.y = uv[it][1];
        v.z = uv[it][2];
        if (kStart == kFromUProlong) {
          const float3 p = cprolong_site(cb, x0 - 1 + lx, y0 - 1 + ly, z0 - 1 + lz, c0x, c0y, c0z);
          v.x += p.x;
          v.y += p.y;
          v.z += p.z;
        }
      }
      csm[csite(lx, ly, lz)] = v;
    }
  }
  __syncthreads();
  CPassOps oa, ob;
  if (!reverse) {
    ctile_step<0, 0, 0, 1, 0, 0>(csm, d, x0, y0, z0, st, f, first, ob);
    __syncthreads();
    ctile_step<1, 0, 0, 0, 1, 0>(csm, d, x0, y0, z0, st, f, ob, oa);
    __syncthreads();
    ctile_step<0, 1, 0, 1, 1, 0>(csm, d, x0, y0, z0, st, f, oa, ob);
    __syncthreads();
    ctile_step<1, 1, 0, 0, 0, 1>(csm, d, x0, y0, z0, st, f, ob, oa);
    __syncthreads();
    ctile_step<0, 0, 1, 1, 0, 1>(csm, d, x0, y0, z0, st, f, oa, ob);
    __syncthreads();
    ctile_step<1, 0, 1, 0, 1, 1>(csm, d, x0, y0, z0, st, f, ob, oa);
    __syncthreads();
    ctile_step<0, 1, 1, 1, 1, 1>(csm, d, x0, y0, z0, st, f, oa, ob);
    __syncthreads();
    ctile_apply<1, 1, 1>(csm, ob);
  } else {
    ctile_step<1, 1, 1, 0, 1, 1>(csm, d, x0, y0, z0, st, f, first, ob);
    __syncthreads();
    ctile_step<0, 1, 1, 1, 0, 1>(csm, d, x0, y0, z0, st, f, ob, oa);
    __syncthreads();
    ctile_step<1, 0, 1, 0, 0, 1>(csm, d, x0, y0, z0, st, f, oa, ob);
    __syncthreads();
    ctile_step<0, 0, 1, 1, 1, 0>(csm, d, x0, y0, z0, st, f, ob, oa);
    __syncthreads();
    ctile_step<1, 1, 0, 0, 1, 0>(csm, d, x0, y0, z0, st, f, oa, ob);
    __syncthreads();
    ctile_step<0, 1, 0, 1, 0, 0>(csm, d, x0, y0, z0, st, f, ob, oa);
    __syncthreads();
    ctile_step<1, 0, 0, 0, 0, 0>(csm, d, x0, y0, z0, st, f, oa, ob);
    __syncthreads();
    ctile_apply<0, 0, 0>(csm, ob);
  }
  __syncthreads();
  for (int s = t; s < kCTX * kCTY * kCTZ; s += kCThreads) {
    const int lx = 1 + s % kCTX, ly = 1 + (s / kCTX) % kCTY, lz = 1 + s / (kCTX * kCTY);
    const float4 o = csm[csite(lx, ly, lz)];
    const size_t g = size_t(wrapm(x0 + lx - 1, d.nx)) +
                     size_t(d.nx) * (size_t(wrapm(y0 + ly - 1, d.ny)) + size_t(d.ny) * wrapm(z0 + lz - 1, d.nz));
    u_out[g] = o.x;
    u_out[nv + g] = o.y;
    u_out[2 * nv + g] = o.z;
  }
}

}  // namespace otm
