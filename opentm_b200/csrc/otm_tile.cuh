// otm_tile.cuh -- tile-staged fine-level smoother and residual (sm_100a).
//
// The fine level's Gauss-Seidel smoothing runs one launch per sweep instead of one launch per
// colour pair: every CTA stages a tile of 16 x 16 x 8 vertices plus a one-site halo in shared
// memory, as one float4 per site {u_case0, u_case1, u_case2, k_e} (k_e the conductivity of the
// element whose lower corner is the site), runs the four colour-pair passes of the sweep inside
// the tile with the halo held at the values it had when the sweep started, and writes the tile's
// interior to a second buffer (so that no tile reads a halo another tile has already overwritten).
// Inside a tile this is the colour-ordered Gauss-Seidel sweep of the reference smoother
// (homogenization/grid.cu:318-471, colours in the order 0,4,1,5,2,6,3,7, the pairs (cx,cy,0) /
// (cx,cy,1) updated together because the cube element couples no vertices one edge apart); across
// tile faces it is block Jacobi. Block Jacobi alone leaves the error that is constant inside each
// tile and alternates in sign from tile to tile nearly undamped, so consecutive sweeps alternate
// between two tilings, the second shifted by half a tile along every axis: the faces of one tiling
// lie inside the tiles of the other. The first sweep after the coarse-grid correction adds the
// trilinear prolongation P u_c while it stages the tile. Pre-smoothing runs forward with the
// tilings 0, 1, 0, ..., post-smoothing in the reverse pair order with the tilings mirrored, so the
// V-cycle stays symmetric (the post leg is the transpose of the pre leg), as PCG needs.
//
// The tile's right-hand side (3 cases, FP32, 24 KB) arrives by TMA tensor copies
// (cp.async.bulk.tensor of eight 4-D boxes {8, 8, 4, 3}, whose periodic origins a shifted tile
// may wrap, completion on one mbarrier) issued at kernel entry, so it lands while the threads
// stage the sites.
//
// Shared-memory layout of the sites: site (lx, ly, lz), lx, ly in [0, 18), lz in [0, 10), lies at
// lz * 342 + ly * 19 + (lx odd ? 9 + lx / 2 : lx / 2): within a row the even and the odd sites are
// stored apart, so that the 8 lanes that update every other site of a row read 8 consecutive
// float4, and rows are padded to 19 float4 so that the rows two apart, which the other lanes of a
// warp read, start in other banks.
//
// A thread owns a column segment of 4 vertices of one colour pair and streams the 6 planes around
// it: every staged plane is read once (8 neighbour sites + the own site's conductivity) and added
// to the three vertices it couples to (the one above, the one in the plane, the one below), so a
// vertex costs about 13 shared-memory loads instead of 28.
#pragma once

#include <cuda.h>

#include "otm_mg_kernels.cuh"

namespace otm {

constexpr int kTX = 16, kTY = 16, kTZ = 8;                    // interior vertices of a tile
constexpr int kSX = kTX + 2, kSY = kTY + 2, kSZ = kTZ + 2;    // staged sites (one halo site each side)
constexpr int kSHalf = kSX / 2;                               // sites of one parity in a row
constexpr int kSRow = kSX + 1;                                // row pitch in float4 (padded)
constexpr int kSPlane = kSRow * kSY;                          // 342
constexpr int kSSites = kSPlane * kSZ;                        // 3420
constexpr int kSmoothThreads = 128;                           // 8 x 8 pair columns x 2 segments
constexpr int kResidThreads = 256;                            // one thread per column
constexpr int kSeg = 4;                                       // vertices per thread and pass
constexpr int kCX = kTX / 2 + 2, kCY = kTY / 2 + 2, kCZ = kTZ / 2 + 2;  // staged coarse sites
constexpr int kCSites = kCX * kCY * kCZ;                      // 600
constexpr int kFElems = 3 * kTX * kTY * kTZ;                  // right-hand side of a tile (6144 floats)
constexpr int kFBX = 8, kFBY = 8, kFBZ = 4;                   // TMA box of the right-hand side (x 3 cases)
constexpr int kFBox = kFBX * kFBY * kFBZ * 3;                 // 768 floats per box
constexpr int kFCase = kFBX * kFBY * kFBZ;                    // case stride inside a box (256)
static_assert((kTX / 2) * (kTY / 2) * (kTZ / kSeg) == kSmoothThreads, "one thread per column segment");
static_assert(kTX * kTY == kResidThreads, "one thread per column");
static_assert(kSeg == kFBZ && kTX == 2 * kFBX && kTY == 2 * kFBY && kTZ == 2 * kFBZ,
              "a column segment lies in one right-hand-side box along z; 2 x 2 x 2 boxes per tile");

// Dynamic shared memory: [right-hand-side boxes][mbarrier][sites][coarse block], after rounding the
// base up to 128 bytes (the TMA destination's alignment).
constexpr size_t kOffBar = size_t(kFElems) * sizeof(float);
constexpr size_t kOffSites = kOffBar + 128;
constexpr size_t kOffCoarse = kOffSites + size_t(kSSites) * sizeof(float4);
constexpr size_t kTileSmemSweep = kOffCoarse + 128;                                      // 79,552 B
constexpr size_t kTileSmemProlong = kOffCoarse + size_t(kCSites) * sizeof(float4) + 128;  // 89,152 B
constexpr size_t kTileSmemResid = kOffCoarse + 128;
constexpr uint32_t kFBytes = uint32_t(kFElems * sizeof(float));

// Polls of the right-hand-side copy's mbarrier before a CTA gives up (each poll may suspend the
// thread for a short hardware-defined time; together well over a second).
constexpr int kTileWaitPolls = 1 << 20;

// Whether a level's dimensions can be tiled.
__host__ __device__ inline bool tile_fits(const Dims& d) {
  return d.nx % kTX == 0 && d.ny % kTY == 0 && d.nz % kTZ == 0;
}
__host__ __device__ inline unsigned tile_count(const Dims& d) {
  return unsigned(d.nx / kTX) * unsigned(d.ny / kTY) * unsigned(d.nz / kTZ);
}

__device__ __forceinline__ int tsite(int lx, int ly, int lz) {
  return lz * kSPlane + ly * kSRow + ((lx & 1) ? kSHalf + (lx >> 1) : (lx >> 1));
}
__device__ __forceinline__ int rsite(int lx, int ly, int lz) { return lz * kSPlane + ly * kSRow + lx; }

// Origin (x0, y0, z0) of tile b of tiling `shift` (0: tiles at multiples of the tile size; 1:
// shifted by half a tile along every axis, so the last tile of a row wraps around the periodic
// cell). Tiles are ordered x fastest so that neighbouring CTAs share halos. The origin is not
// wrapped: global indices of the tile's sites are.
__device__ __forceinline__ void tile_origin(const Dims& d, unsigned b, int shift, int& x0, int& y0, int& z0) {
  const unsigned ntx = unsigned(d.nx / kTX), nty = unsigned(d.ny / kTY);
  const unsigned q = b / ntx;
  x0 = int(b - q * ntx) * kTX + shift * (kTX / 2);
  y0 = int(q % nty) * kTY + shift * (kTY / 2);
  z0 = int(q / nty) * kTZ + shift * (kTZ / 2);
}

// Position of the right-hand side of tile vertex (x, y, z) (0-based inside the tile) of case 0 in
// the staged boxes; case c is kFCase further: box (x / 8, y / 8, z / 4), inside it x, y, z, case.
__device__ __forceinline__ int fpos(int x, int y, int z) {
  return ((x >> 3) + 2 * (y >> 3) + 4 * (z >> 2)) * kFBox + ((z & 3) * kFBY + (y & 7)) * kFBX + (x & 7);
}

// ---- the right-hand-side copy: TMA tensor loads completing on an mbarrier ---------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Thread 0 initialises the barrier and starts the copies of the tile's right-hand side (eight
// boxes, their periodic origins wrapped; an origin is a multiple of 8 (x, y) or 4 (z) and the
// level's dimensions are multiples of 16 and 8, so no box crosses the periodic boundary). The
// barrier initialisation is published to the other threads by the __syncthreads() that precedes
// the wait.
__device__ __forceinline__ void tile_f_copy_start(const CUtensorMap* fmap, float* fsm, uint64_t* bar, const Dims& d,
                                                  int x0, int y0, int z0) {
  if (threadIdx.x == 0) {
    const uint32_t b = smem_addr(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(b), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(kFBytes) : "memory");
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int X = wrapm(x0 + kFBX * (q & 1), d.nx), Y = wrapm(y0 + kFBY * ((q >> 1) & 1), d.ny),
                Z = wrapm(z0 + kFBZ * (q >> 2), d.nz);
      asm volatile(
          "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
          "%4, %5}], [%6];" ::"r"(smem_addr(fsm + q * kFBox)),
          "l"(reinterpret_cast<uint64_t>(fmap)), "r"(X), "r"(Y), "r"(Z), "r"(0), "r"(b)
          : "memory");
    }
  }
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the copies. One thread polls the mbarrier (polls by every thread would compete
// with the other CTA's passes for shared-memory bandwidth and issue slots); the others wait at the
// barrier, which also makes the copied data visible to them. Returns false in every thread of the
// CTA if the polls ran out; then the solve is flagged (timeout + done) and the polling thread waits
// once more, again bounded, for the copies it issued before the CTA returns.
__device__ __forceinline__ bool tile_f_copy_wait(uint64_t* bar, SolveScalars* sc) {
  bool ok = true;
  if (threadIdx.x == 0) {
    ok = false;
    for (int i = 0; i < kTileWaitPolls && !ok; i++) ok = mbar_try_wait(bar, 0);
    if (!ok) {
      if (sc) {
        atomicExch(&sc->timeout, 1);
        atomicExch(&sc->done, 1);
      }
      for (int i = 0; i < kTileWaitPolls && !ok; i++) ok = mbar_try_wait(bar, 0);
      ok = false;
    }
  }
  return !__syncthreads_or(!ok);
}

// ---- vector loads and stores of 4 consecutive values in the storage types --------------------
__device__ __forceinline__ void ld4(const float* p, float (&v)[4]) {
  const float4 q = __ldg(reinterpret_cast<const float4*>(p));
  v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
}
__device__ __forceinline__ void ld4(const __nv_bfloat16* p, float (&v)[4]) {
  const uint2 q = __ldg(reinterpret_cast<const uint2*>(p));
  const __nv_bfloat162 a = *reinterpret_cast<const __nv_bfloat162*>(&q.x);
  const __nv_bfloat162 b = *reinterpret_cast<const __nv_bfloat162*>(&q.y);
  v[0] = __low2float(a), v[1] = __high2float(a), v[2] = __low2float(b), v[3] = __high2float(b);
}
__device__ __forceinline__ void ld4(const __half* p, float (&v)[4]) {
  const uint2 q = __ldg(reinterpret_cast<const uint2*>(p));
  const __half2 a = *reinterpret_cast<const __half2*>(&q.x);
  const __half2 b = *reinterpret_cast<const __half2*>(&q.y);
  v[0] = __low2float(a), v[1] = __high2float(a), v[2] = __low2float(b), v[3] = __high2float(b);
}
__device__ __forceinline__ void st4(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ void st4(__nv_bfloat16* p, const float (&v)[4]) {
  const __nv_bfloat162 a = __floats2bfloat162_rn(v[0], v[1]), b = __floats2bfloat162_rn(v[2], v[3]);
  uint2 q;
  q.x = *reinterpret_cast<const uint32_t*>(&a);
  q.y = *reinterpret_cast<const uint32_t*>(&b);
  *reinterpret_cast<uint2*>(p) = q;
}
__device__ __forceinline__ void st4(__half* p, const float (&v)[4]) {
  const __half2 a = __floats2half2_rn(v[0], v[1]), b = __floats2half2_rn(v[2], v[3]);
  uint2 q;
  q.x = *reinterpret_cast<const uint32_t*>(&a);
  q.y = *reinterpret_cast<const uint32_t*>(&b);
  *reinterpret_cast<uint2*>(p) = q;
}

// ---- coefficients ------------------------------------------------------------------------------
// Coefficients of the 8 neighbour columns of a vertex for one element plane, from the 4
// conductivities K[b] (b = bx + 2 by: the element whose lower corner is (x - 1 + bx, y - 1 + by)
// in that plane). Neighbour n: 0 (-1,-1) 1 (0,-1) 2 (+1,-1) 3 (-1,0) 4 (+1,0) 5 (-1,+1) 6 (0,+1)
// 7 (+1,+1). Corners couple through one element of the plane (c3, three axes apart), the four
// edge neighbours through two (c2, two axes apart): A(v, v+o) = c[|o|_0] * sum of the
// conductivities of the elements holding both vertices.
struct PlaneCoef {
  float w[8];
  __device__ __forceinline__ void make(const float (&K)[4], const FineOp& op) {
    w[0] = op.c3 * K[0];
    w[1] = op.c2 * (K[0] + K[1]);
    w[2] = op.c3 * K[1];
    w[3] = op.c2 * (K[0] + K[2]);
    w[4] = op.c2 * (K[1] + K[3]);
    w[5] = op.c3 * K[2];
    w[6] = op.c2 * (K[2] + K[3]);
    w[7] = op.c3 * K[3];
  }
};

// acc -= sum_n w[n] * nb[n] (3 cases)
__device__ __forceinline__ void sub_plane(float (&acc)[3], const PlaneCoef& c, const float4 (&nb)[8]) {
#pragma unroll
  for (int n = 0; n < 8; n++) {
    acc[0] -= c.w[n] * nb[n].x;
    acc[1] -= c.w[n] * nb[n].y;
    acc[2] -= c.w[n] * nb[n].z;
  }
}

// in-plane corners of the vertex in the plane: c2 * (K_below + K_above) per corner
__device__ __forceinline__ void sub_inplane(float (&acc)[3], const float (&Kb)[4], const float (&Ka)[4],
                                            const FineOp& op, const float4 (&nb)[8]) {
  const int cn[4] = {0, 2, 5, 7};
#pragma unroll
  for (int b = 0; b < 4; b++) {
    const float w = op.c2 * (Kb[b] + Ka[b]);
    acc[0] -= w * nb[cn[b]].x;
    acc[1] -= w * nb[cn[b]].y;
    acc[2] -= w * nb[cn[b]].z;
  }
}

// One colour-pair pass (PX, PY) over the tile's interior: every thread updates the 4 vertices
// (lx, ly, lz0 .. lz0 + 3) of its column segment, reading planes lz0 - 1 .. lz0 + 4. fsm holds the
// staged right-hand side (see fpos), fs the per-case scale applied to it.
template <int PX, int PY>
__device__ __forceinline__ void tile_pass(float4* sm, const float* fsm, const FineOp& op, const float (&fs)[3]) {
  const int t = int(threadIdx.x);
  const int i = t & 7, j = (t >> 3) & 7, seg = t >> 6;
  const int lx = 2 * i + 1 + PX, ly = 2 * j + 1 + PY, lz0 = 1 + kSeg * seg;
  // positions of the left / right neighbour columns relative to the own site: the parity of lx
  // is fixed by the pass, so they are compile-time offsets in the parity-split row
  constexpr int oL = PX ? kSHalf - 1 : -kSHalf, oR = PX ? kSHalf : -kSHalf + 1;
  const float* fcol = fsm + fpos(lx - 1, ly - 1, lz0 - 1);  // vertex q of the segment: + q * 64
  float Kp[4] = {0.f, 0.f, 0.f, 0.f};  // conductivities of the previous plane
  PlaneCoef Cp;                        // coefficients of the previous plane
  float accA[3] = {0.f, 0.f, 0.f}, accB[3] = {0.f, 0.f, 0.f}, accC[3] = {0.f, 0.f, 0.f};  // P-1, P, P+1
  float dA = 0.f, dB = 0.f;  // their conductivity sums so far
#pragma unroll
  for (int s = 0; s < kSeg + 2; s++) {
    const int P = lz0 - 1 + s;
    const float4* b = sm + tsite(lx, ly, P);
    float4 nb[8];
    nb[0] = b[oL - kSRow];
    nb[1] = b[-kSRow];
    nb[2] = b[oR - kSRow];
    nb[3] = b[oL];
    nb[4] = b[oR];
    nb[5] = b[oL + kSRow];
    nb[6] = b[kSRow];
    nb[7] = b[oR + kSRow];
    const float kown = reinterpret_cast<const float*>(b)[3];
    const float K[4] = {nb[0].w, nb[1].w, nb[3].w, kown};
    const float sK = (K[0] + K[1]) + (K[2] + K[3]);
    PlaneCoef C;
    C.make(K, op);
    // vertex P + 1 (segment index s): its lower element plane is P
    float dC = 0.f;
    if (s < kSeg) {
      const float* fv = fcol + s * (kFBX * kFBY);
#pragma unroll
      for (int c = 0; c < 3; c++) accC[c] = fv[c * kFCase] * fs[c];
      sub_plane(accC, C, nb);
      dC = sK;
    }
    // vertex P (index s - 1): in-plane corners, elements of planes P - 1 and P
    if (s >= 1 && s <= kSeg) {
      sub_inplane(accB, Kp, K, op, nb);
      dB += sK;
    }
    // vertex P - 1 (index s - 2): its upper element plane is P - 1; complete now
    if (s >= 2) {
      sub_plane(accA, Cp, nb);
      const float inv = 1.0f / (op.c0 * dA);
      float4 o;
      o.x = accA[0] * inv;
      o.y = accA[1] * inv;
      o.z = accA[2] * inv;
      o.w = Kp[3];  // own element of plane P - 1
      sm[tsite(lx, ly, P - 1)] = o;
    }
    // rotate: P becomes P - 1, P + 1 becomes P
#pragma unroll
    for (int c = 0; c < 3; c++) {
      accA[c] = accB[c];
      accB[c] = accC[c];
    }
    dA = dB;
    dB = dC;
#pragma unroll
    for (int q = 0; q < 4; q++) Kp[q] = K[q];
    Cp = C;
  }
}

// Trilinear prolongation of the staged coarse block (float4 per coarse site, cases in x, y, z) at
// the fine site with unwrapped coordinates (ux, uy, uz); c0x/c0y/c0z are the coarse coordinates
// of the block's first site. The expression and weights are those of prolong_body.
__device__ __forceinline__ float3 prolong_site(const float4* cb, int ux, int uy, int uz, int c0x, int c0y, int c0z) {
  const int ax0 = (ux >> 1) - c0x, ay0 = (uy >> 1) - c0y, az0 = (uz >> 1) - c0z;
  const int ax1 = ax0 + (ux & 1), ay1 = ay0 + (uy & 1), az1 = az0 + (uz & 1);
  const float wx1 = (ux & 1) ? 0.5f : 0.f, wy1 = (uy & 1) ? 0.5f : 0.f, wz1 = (uz & 1) ? 0.5f : 0.f;
  const float wx0 = 1.f - wx1, wy0 = 1.f - wy1, wz0 = 1.f - wz1;
  const float4* r00 = cb + (ay0 + kCY * az0) * kCX;
  const float4* r10 = cb + (ay1 + kCY * az0) * kCX;
  const float4* r01 = cb + (ay0 + kCY * az1) * kCX;
  const float4* r11 = cb + (ay1 + kCY * az1) * kCX;
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

// The prolongation at the 4 fine sites xs .. xs + 3 of a row (xs even, unwrapped), reading the 3
// coarse columns under them once per coarse row instead of 8 coarse sites per fine site. The
// trilinear weights are separable: each coarse column is first interpolated over (y, z), then the
// even sites take their column's value and the odd ones the mean of two columns (the weights of
// prolong_site, summed in another order).
__device__ __forceinline__ void prolong_quad(const float4* cb, int xs, int uy, int uz, int c0x, int c0y, int c0z,
                                             float3 (&o)[4]) {
  const int ax = (xs >> 1) - c0x;  // coarse columns ax, ax + 1, ax + 2
  const int ay0 = (uy >> 1) - c0y, az0 = (uz >> 1) - c0z;
  const int ay1 = ay0 + (uy & 1), az1 = az0 + (uz & 1);
  const float wy1 = (uy & 1) ? 0.5f : 0.f, wz1 = (uz & 1) ? 0.5f : 0.f;
  const float wy0 = 1.f - wy1, wz0 = 1.f - wz1;
  const float4* rows[4] = {cb + (ay0 + kCY * az0) * kCX + ax, cb + (ay1 + kCY * az0) * kCX + ax,
                           cb + (ay0 + kCY * az1) * kCX + ax, cb + (ay1 + kCY * az1) * kCX + ax};
  float3 col[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const float4 v0 = rows[0][a], v1 = rows[1][a], v2 = rows[2][a], v3 = rows[3][a];
    col[a].x = wz0 * (wy0 * v0.x + wy1 * v1.x) + wz1 * (wy0 * v2.x + wy1 * v3.x);
    col[a].y = wz0 * (wy0 * v0.y + wy1 * v1.y) + wz1 * (wy0 * v2.y + wy1 * v3.y);
    col[a].z = wz0 * (wy0 * v0.z + wy1 * v1.z) + wz1 * (wy0 * v2.z + wy1 * v3.z);
  }
  o[0] = col[0];
  o[1] = make_float3(0.5f * (col[0].x + col[1].x), 0.5f * (col[0].y + col[1].y), 0.5f * (col[0].z + col[1].z));
  o[2] = col[1];
  o[3] = make_float3(0.5f * (col[1].x + col[2].x), 0.5f * (col[1].y + col[2].y), 0.5f * (col[1].z + col[2].z));
}

// Stages the tile's sites {u_case0, u_case1, u_case2, k_e} in shared memory (parity-split order
// when kSplit, natural order otherwise). With kWithU the values are u (and, when uc is given, plus
// the trilinear prolongation of the coarse correction uc, whose block under the tile is staged in
// cb first); without it they start at 0. Every thread first issues all its global loads (4 values
// of a row at a time for the interior, single values for the two halo columns and the coarse
// block) and only then stores, so a CTA waits for one round of memory latency, not one per site.
template <bool kWithU, int NT, bool kSplit, typename KT, typename VT>
__device__ __forceinline__ void stage_tile(const Dims& d, const Dims& dc, int x0, int y0, int z0,
                                           const KT* __restrict__ ks, const VT* __restrict__ u,
                                           const float* __restrict__ uc, float4* sm, float4* cb) {
  constexpr int kQuads = kSY * kSZ * (kTX / 4), kQI = (kQuads + NT - 1) / NT;
  constexpr int kHalo = kSY * kSZ * 2, kHI = (kHalo + NT - 1) / NT;
  constexpr int kCI = (kCSites + NT - 1) / NT;
  const int t = int(threadIdx.x);
  const size_t nv = d.nv();
  const int c0x = x0 / 2 - 1, c0y = y0 / 2 - 1, c0z = z0 / 2 - 1;
  const bool prolong = kWithU && uc != nullptr;
  // 1. all loads
  float cbv[kCI][3];
  if (prolong) {
    const size_t nvc = dc.nv();
#pragma unroll
    for (int it = 0; it < kCI; it++) {
      const int s = t + it * NT;
      if (s < kCSites) {
        const int ax = s % kCX, ay = (s / kCX) % kCY, az = s / (kCX * kCY);
        const int X = wrapm(c0x + ax, dc.nx), Y = wrapm(c0y + ay, dc.ny), Z = wrapm(c0z + az, dc.nz);
        const size_t g = size_t(X) + size_t(dc.nx) * (size_t(Y) + size_t(dc.ny) * Z);
#pragma unroll
        for (int c = 0; c < 3; c++) cbv[it][c] = __ldg(uc + c * nvc + g);
      }
    }
  }
  float kq[kQI][4], uq[kWithU ? kQI : 1][3][4];
#pragma unroll
  for (int it = 0; it < kQI; it++) {
    const int w = t + it * NT;
    if (w < kQuads) {
      const int q = w & 3, row = w >> 2;
      const int ly = row % kSY, lz = row / kSY;
      const size_t g = size_t(wrapm(x0 + 4 * q, d.nx)) +
                       size_t(d.nx) * (size_t(wrapm(y0 - 1 + ly, d.ny)) + size_t(d.ny) * wrapm(z0 - 1 + lz, d.nz));
      ld4(ks + g, kq[it]);
      if (kWithU)
#pragma unroll
        for (int c = 0; c < 3; c++) ld4(u + c * nv + g, uq[it][c]);
    }
  }
  float kh[kHI], uh[kWithU ? kHI : 1][3];
#pragma unroll
  for (int it = 0; it < kHI; it++) {
    const int w = t + it * NT;
    if (w < kHalo) {
      const int side = w & 1, row = w >> 1;
      const int ly = row % kSY, lz = row / kSY;
      const int lx = side ? kSX - 1 : 0;
      const size_t g = size_t(wrapm(x0 - 1 + lx, d.nx)) +
                       size_t(d.nx) * (size_t(wrapm(y0 - 1 + ly, d.ny)) + size_t(d.ny) * wrapm(z0 - 1 + lz, d.nz));
      kh[it] = ld(ks + g);
      if (kWithU)
#pragma unroll
        for (int c = 0; c < 3; c++) uh[it][c] = ld(u + c * nv + g);
    }
  }
  // 2. the coarse block, needed by every thread's prolongation
  if (prolong) {
#pragma unroll
    for (int it = 0; it < kCI; it++) {
      const int s = t + it * NT;
      if (s < kCSites) cb[s] = make_float4(cbv[it][0], cbv[it][1], cbv[it][2], 0.f);
    }
    __syncthreads();
  }
  // 3. the sites
#pragma unroll
  for (int it = 0; it < kQI; it++) {
    const int w = t + it * NT;
    if (w < kQuads) {
      const int q = w & 3, row = w >> 2;
      const int ly = row % kSY, lz = row / kSY;
      float3 p[4] = {};
      if (prolong) prolong_quad(cb, x0 + 4 * q, y0 - 1 + ly, z0 - 1 + lz, c0x, c0y, c0z, p);
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int lx = 1 + 4 * q + e;
        float4 v = make_float4(0.f, 0.f, 0.f, kq[it][e]);
        if (kWithU) {
          v.x = uq[it][0][e];
          v.y = uq[it][1][e];
          v.z = uq[it][2][e];
          if (prolong) {
            v.x += p[e].x;
            v.y += p[e].y;
            v.z += p[e].z;
          }
        }
        sm[kSplit ? tsite(lx, ly, lz) : rsite(lx, ly, lz)] = v;
      }
    }
  }
#pragma unroll
  for (int it = 0; it < kHI; it++) {
    const int w = t + it * NT;
    if (w < kHalo) {
      const int side = w & 1, row = w >> 1;
      const int ly = row % kSY, lz = row / kSY;
      const int lx = side ? kSX - 1 : 0;
      float4 v = make_float4(0.f, 0.f, 0.f, kh[it]);
      if (kWithU) {
        v.x = uh[it][0];
        v.y = uh[it][1];
        v.z = uh[it][2];
        if (prolong) {
          const float3 p = prolong_site(cb, x0 - 1 + lx, y0 - 1 + ly, z0 - 1 + lz, c0x, c0y, c0z);
          v.x += p.x;
          v.y += p.y;
          v.z += p.z;
        }
      }
      sm[kSplit ? tsite(lx, ly, lz) : rsite(lx, ly, lz)] = v;
    }
  }
}

// Aligned base of the dynamic shared memory (128 bytes: the TMA destination).
__device__ __forceinline__ unsigned char* tile_smem_base() {
  extern __shared__ unsigned char tile_smem_raw[];
  const uintptr_t a = reinterpret_cast<uintptr_t>(tile_smem_raw);
  return reinterpret_cast<unsigned char*>((a + 127) & ~uintptr_t(127));
}

// Start of a sweep: from zero (the first pre-smoothing sweep), from u_in, or from u_in plus the
// trilinear prolongation of the coarse correction (the first post-smoothing sweep).
enum TileStart { kFromZero = 0, kFromU = 1, kFromUProlong = 2 };

// One Gauss-Seidel sweep of the fine level on the tiles of tiling `shift` (see above): the tile is
// staged from the start values (kStart), the four colour-pair passes run in the order 0,1,2,3, or
// 3,2,1,0 when `reverse`, and the interior goes to u_out, which must not alias u_in. ks: fine
// conductivity (storage KT); fmap: TMA map of the right-hand side (FP32, 3 cases, scaled per case
// by fscale when given); u_in / u_out in storage VT; uc: the coarse correction (FP32, kFromUProlong,
// homogenization/grid.cu:881-940); arithmetic and shared memory FP32.
template <int kStart, typename KT, typename VT>
__global__ void __launch_bounds__(kSmoothThreads, 2)
    k_tile_sweep(const __grid_constant__ CUtensorMap fmap, Dims d, Dims dc, const KT* __restrict__ ks, FineOp op,
                 const VT* __restrict__ u_in, const float* __restrict__ uc, VT* __restrict__ u_out,
                 const double* fscale, int shift, int reverse, SolveScalars* sc) {
  unsigned char* base = tile_smem_base();
  float* fsm = reinterpret_cast<float*>(base);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + kOffBar);
  float4* sm = reinterpret_cast<float4*>(base + kOffSites);
  float4* cb = reinterpret_cast<float4*>(base + kOffCoarse);
  pdl_wait();
  if (sc && solve_done(sc)) return;
  int x0, y0, z0;
  tile_origin(d, blockIdx.x, shift, x0, y0, z0);
  const size_t nv = d.nv();
  tile_f_copy_start(&fmap, fsm, bar, d, x0, y0, z0);
  float fs[3] = {1.f, 1.f, 1.f};
  if (fscale)
#pragma unroll
    for (int c = 0; c < 3; c++) fs[c] = float(fscale[c]);
  stage_tile<kStart != kFromZero, kSmoothThreads, true>(d, dc, x0, y0, z0, ks, u_in,
                                                        kStart == kFromUProlong ? uc : nullptr, sm, cb);
  __syncthreads();
  if (!tile_f_copy_wait(bar, sc)) return;
  if (!reverse) {
    tile_pass<0, 0>(sm, fsm, op, fs);
    __syncthreads();
    tile_pass<1, 0>(sm, fsm, op, fs);
    __syncthreads();
    tile_pass<0, 1>(sm, fsm, op, fs);
    __syncthreads();
    tile_pass<1, 1>(sm, fsm, op, fs);
  } else {
    tile_pass<1, 1>(sm, fsm, op, fs);
    __syncthreads();
    tile_pass<0, 1>(sm, fsm, op, fs);
    __syncthreads();
    tile_pass<1, 0>(sm, fsm, op, fs);
    __syncthreads();
    tile_pass<0, 0>(sm, fsm, op, fs);
  }
  __syncthreads();
  // interior to global memory, 4 consecutive x at a time
  for (int w = int(threadIdx.x); w < kTX * kTY * kTZ / 4; w += kSmoothThreads) {
    const int q = w & 3, row = w >> 2;
    const int ly = 1 + row % kTY, lz = 1 + row / kTY;
    float o0[4], o1[4], o2[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float4 v = sm[tsite(1 + 4 * q + e, ly, lz)];
      o0[e] = v.x, o1[e] = v.y, o2[e] = v.z;
    }
    const size_t g = size_t(wrapm(x0 + 4 * q, d.nx)) +
                     size_t(d.nx) * (size_t(wrapm(y0 + ly - 1, d.ny)) + size_t(d.ny) * size_t(wrapm(z0 + lz - 1, d.nz)));
    st4(u_out + g, o0);
    st4(u_out + nv + g, o1);
    st4(u_out + 2 * nv + g, o2);
  }
}

// r = f - A u on the fine level for every vertex of a tile (tiling 0), from a staged tile with its
// halo (natural site order here: lanes take consecutive sites of a row). A thread owns one column
// of the tile and streams its 10 planes.
template <typename KT, typename VT>
__global__ void __launch_bounds__(kResidThreads, 2)
    k_tile_resid(const __grid_constant__ CUtensorMap fmap, Dims d, const KT* __restrict__ ks, FineOp op,
                 const VT* __restrict__ u, VT* __restrict__ r, const double* fscale, SolveScalars* sc) {
  unsigned char* base = tile_smem_base();
  float* fsm = reinterpret_cast<float*>(base);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + kOffBar);
  float4* sm = reinterpret_cast<float4*>(base + kOffSites);
  pdl_wait();
  if (sc && solve_done(sc)) return;
  int x0, y0, z0;
  tile_origin(d, blockIdx.x, 0, x0, y0, z0);
  const size_t nv = d.nv();
  tile_f_copy_start(&fmap, fsm, bar, d, x0, y0, z0);
  float fs[3] = {1.f, 1.f, 1.f};
  if (fscale)
#pragma unroll
    for (int c = 0; c < 3; c++) fs[c] = float(fscale[c]);
  stage_tile<true, kResidThreads, false>(d, d, x0, y0, z0, ks, u, (const float*)nullptr, sm, (float4*)nullptr);
  __syncthreads();
  if (!tile_f_copy_wait(bar, sc)) return;
  const int lx = 1 + (int(threadIdx.x) & 15), ly = 1 + (int(threadIdx.x) >> 4);
  const size_t col = size_t(x0 + lx - 1) + size_t(d.nx) * size_t(y0 + ly - 1);
  const size_t pl = size_t(d.nx) * d.ny;
  float Kp[4] = {0.f, 0.f, 0.f, 0.f};
  PlaneCoef Cp;
  float accA[3] = {0.f, 0.f, 0.f}, accB[3] = {0.f, 0.f, 0.f}, accC[3] = {0.f, 0.f, 0.f};
  float dA = 0.f, dB = 0.f;
  float uA[3] = {0.f, 0.f, 0.f}, uB[3] = {0.f, 0.f, 0.f};  // own values of the vertices P - 1, P
#pragma unroll 1
  for (int P = 0; P < kSZ; P++) {
    const float4* b = sm + rsite(lx, ly, P);
    float4 nb[8];
    nb[0] = b[-kSRow - 1];
    nb[1] = b[-kSRow];
    nb[2] = b[-kSRow + 1];
    nb[3] = b[-1];
    nb[4] = b[1];
    nb[5] = b[kSRow - 1];
    nb[6] = b[kSRow];
    nb[7] = b[kSRow + 1];
    const float4 own = b[0];
    const float K[4] = {nb[0].w, nb[1].w, nb[3].w, own.w};
    const float sK = (K[0] + K[1]) + (K[2] + K[3]);
    PlaneCoef C;
    C.make(K, op);
    float dC = 0.f;
    // vertex P + 1 (interior planes 1..8): lower element plane P
    if (P + 1 <= kTZ) {
      const float* fv = fsm + fpos(lx - 1, ly - 1, P);
#pragma unroll
      for (int c = 0; c < 3; c++) accC[c] = fv[c * kFCase] * fs[c];
      sub_plane(accC, C, nb);
      dC = sK;
    }
    // vertex P: in-plane corners and its own value
    if (P >= 1 && P <= kTZ) {
      sub_inplane(accB, Kp, K, op, nb);
      dB += sK;
      uB[0] = own.x;
      uB[1] = own.y;
      uB[2] = own.z;
    }
    // vertex P - 1: upper element plane P - 1, then r = f - offdiag - diag u
    if (P >= 2) {
      sub_plane(accA, Cp, nb);
      const float diag = op.c0 * dA;
      const size_t g = col + size_t(z0 + P - 2) * pl;
      st(r + g, accA[0] - diag * uA[0]);
      st(r + nv + g, accA[1] - diag * uA[1]);
      st(r + 2 * nv + g, accA[2] - diag * uA[2]);
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      accA[c] = accB[c];
      accB[c] = accC[c];
      uA[c] = uB[c];
    }
    dA = dB;
    dB = dC;
#pragma unroll
    for (int q = 0; q < 4; q++) Kp[q] = K[q];
    Cp = C;
  }
}

// The PCG direction update and operator product of k_update_p_apply_dot on tiles (FP32, cube
// elements): p = (z - zbar) + beta p, q = A z + beta q (A p = A z + beta A p_old, A annihilating
// constants), and the p . q partial sums of the tile, reduced by the last CTA into alpha = rho /
// (p . q). z is staged like u in k_tile_resid (tiling 0, one thread per column streaming its 10
// planes) so its 20 neighbours come from shared memory; beta == 0 (the first iteration) ignores
// the old p and q. part: 3 doubles per tile.
static __global__ void __launch_bounds__(kResidThreads, 2)
    k_tile_apply_dot(Dims d, const float* __restrict__ ks, FineOp op, const float* __restrict__ z,
                     float* __restrict__ p, float* __restrict__ q, double* part, SolveScalars* sc) {
  unsigned char* base = tile_smem_base();
  float4* sm = reinterpret_cast<float4*>(base + kOffSites);
  pdl_wait();
  if (solve_done(sc)) return;
  int x0, y0, z0;
  tile_origin(d, blockIdx.x, 0, x0, y0, z0);
  const size_t nv = d.nv();
  float be[3], zb[3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    be[c] = float(sc->beta[c]);
    zb[c] = float(sc->zmean[c]);
  }
  stage_tile<true, kResidThreads, false>(d, d, x0, y0, z0, ks, z, (const float*)nullptr, sm, (float4*)nullptr);
  __syncthreads();
  const int lx = 1 + (int(threadIdx.x) & 15), ly = 1 + (int(threadIdx.x) >> 4);
  const size_t col = size_t(x0 + lx - 1) + size_t(d.nx) * size_t(y0 + ly - 1);
  const size_t pl = size_t(d.nx) * d.ny;
  float Kp[4] = {0.f, 0.f, 0.f, 0.f};
  PlaneCoef Cp;
  // minus the off-diagonal sums of the vertices P - 1, P, P + 1
  float accA[3] = {0.f, 0.f, 0.f}, accB[3] = {0.f, 0.f, 0.f}, accC[3] = {0.f, 0.f, 0.f};
  float dA = 0.f, dB = 0.f;
  float uA[3] = {0.f, 0.f, 0.f}, uB[3] = {0.f, 0.f, 0.f};  // z of the vertices P - 1, P
  double v[3] = {0, 0, 0};
#pragma unroll 1
  for (int P = 0; P < kSZ; P++) {
    const float4* b = sm + rsite(lx, ly, P);
    float4 nb[8];
    nb[0] = b[-kSRow - 1];
    nb[1] = b[-kSRow];
    nb[2] = b[-kSRow + 1];
    nb[3] = b[-1];
    nb[4] = b[1];
    nb[5] = b[kSRow - 1];
    nb[6] = b[kSRow];
    nb[7] = b[kSRow + 1];
    const float4 own = b[0];
    const float K[4] = {nb[0].w, nb[1].w, nb[3].w, own.w};
    const float sK = (K[0] + K[1]) + (K[2] + K[3]);
    PlaneCoef C;
    C.make(K, op);
    float dC = 0.f;
    if (P + 1 <= kTZ) {  // vertex P + 1: lower element plane P
#pragma unroll
      for (int c = 0; c < 3; c++) accC[c] = 0.f;
      sub_plane(accC, C, nb);
      dC = sK;
    }
    if (P >= 1 && P <= kTZ) {  // vertex P: in-plane corners and its own value
      sub_inplane(accB, Kp, K, op, nb);
      dB += sK;
      uB[0] = own.x;
      uB[1] = own.y;
      uB[2] = own.z;
    }
    if (P >= 2) {  // vertex P - 1: upper element plane P - 1, then the update
      sub_plane(accA, Cp, nb);
      const float diag = op.c0 * dA;
      const size_t g = col + size_t(z0 + P - 2) * pl;
      float po[3], qo[3];  // all loads of the vertex before its stores
#pragma unroll
      for (int c = 0; c < 3; c++) {
        po[c] = be[c] != 0.f ? p[c * nv + g] : 0.f;
        qo[c] = be[c] != 0.f ? q[c * nv + g] : 0.f;
      }
#pragma unroll
      for (int c = 0; c < 3; c++) {
        float pc = uA[c] - zb[c], qc = diag * uA[c] - accA[c];  // accA = -(off-diagonal sum)
        if (be[c] != 0.f) {
          pc += be[c] * po[c];
          qc += be[c] * qo[c];
        }
        p[c * nv + g] = pc;
        q[c * nv + g] = qc;
        v[c] += double(pc) * qc;
      }
    }
#pragma unroll
    for (int c = 0; c < 3; c++) {
      accA[c] = accB[c];
      accB[c] = accC[c];
      uA[c] = uB[c];
    }
    dA = dB;
    dB = dC;
#pragma unroll
    for (int q4 = 0; q4 < 4; q4++) Kp[q4] = K[q4];
    Cp = C;
  }
  double* red = reinterpret_cast<double*>(sm);  // the tile is no longer read
  __syncthreads();
  block_reduce_f64<3>(v, red);
  if (threadIdx.x == 0)
#pragma unroll
    for (int i = 0; i < 3; i++) part[size_t(blockIdx.x) * 3 + i] = v[i];
  if (last_block(&sc->counter[T_PQ])) {
    double t[3];
    reduce_partials<3>(part, int(gridDim.x), t, red);
    if (threadIdx.x == 0) {
      for (int c = 0; c < 3; c++) sc->alpha[c] = t[c] != 0.0 ? sc->rz[c] / t[c] : 0.0;
      sc->counter[T_PQ] = 0;
    }
  }
}

}  // namespace otm
