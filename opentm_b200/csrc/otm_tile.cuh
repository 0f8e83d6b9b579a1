// otm_tile.cuh -- tile-staged fine-level smoother and residual (sm_100a).
//
// The fine level's Gauss-Seidel smoothing runs one launch per smoothing leg instead of one
// launch per colour pair: every CTA stages a tile of 16 x 16 x 8 vertices plus a one-site halo in
// shared memory, as one float4 per site {u_case0, u_case1, u_case2, k_e} (k_e the conductivity of
// the element whose lower corner is the site), runs all colour-pair passes of all sweeps of the leg
// inside the tile with the halo held at the values it had when the leg started, and writes the
// tile's interior back once. Inside a tile this is the colour-ordered Gauss-Seidel sweep of the
// reference smoother (homogenization/grid.cu:318-471, colours in the order 0,4,1,5,2,6,3,7, the
// pairs (cx,cy,0)/(cx,cy,1) updated together because the cube element couples no vertices one
// edge apart); across tile faces it is block Jacobi (hybrid Gauss-Seidel). The leg after the
// coarse-grid correction adds the trilinear prolongation P u_c while it stages the tile and
// writes its result to a second buffer, so that no tile reads a halo another tile has already
// overwritten. Pre-smoothing forward, post-smoothing in the reverse pair order: the V-cycle stays
// symmetric (the post leg's smoother is the transpose of the pre leg's), as PCG needs.
//
// The tile's right-hand side (3 cases, FP32, 24 KB) arrives by one TMA tensor copy
// (cp.async.bulk.tensor, a 4-D box {16, 16, 8, 3} of the level's right-hand side, completion on an
// mbarrier) issued at kernel entry, so it lands while the threads stage the sites.
//
// Shared-memory layout of the sites: site (lx, ly, lz), lx, ly in [0, 18), lz in [0, 10), lies at
// lz * 324 + ly * 18 + (lx odd ? 9 + lx / 2 : lx / 2): within a row the even and the odd sites
// are stored apart, so that the 8 lanes of a quarter warp, which update every other site of a row,
// read 8 consecutive float4 (one 128-byte wavefront, no bank conflict).
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
constexpr int kSPlane = kSX * kSY;                            // 324
constexpr int kSSites = kSPlane * kSZ;                        // 3240
constexpr int kSmoothThreads = 128;                           // 8 x 8 pair columns x 2 segments
constexpr int kResidThreads = 256;                            // one thread per column
constexpr int kSeg = 4;                                       // vertices per thread and pass
constexpr int kCX = kTX / 2 + 2, kCY = kTY / 2 + 2, kCZ = kTZ / 2 + 2;  // staged coarse sites
constexpr int kCSites = kCX * kCY * kCZ;                      // 600
constexpr int kFElems = 3 * kTX * kTY * kTZ;                  // right-hand-side box (6144 floats)
static_assert((kTX / 2) * (kTY / 2) * (kTZ / kSeg) == kSmoothThreads, "one thread per column segment");
static_assert(kTX * kTY == kResidThreads, "one thread per column");

// Dynamic shared memory: [right-hand-side box][mbarrier][sites][coarse block (post leg)], after
// rounding the base up to 128 bytes (the TMA destination's alignment).
constexpr size_t kOffBar = size_t(kFElems) * sizeof(float);
constexpr size_t kOffSites = kOffBar + 128;
constexpr size_t kOffCoarse = kOffSites + size_t(kSSites) * sizeof(float4);
constexpr size_t kTileSmemPre = kOffCoarse + 128;                                      // 76,672 B
constexpr size_t kTileSmemPost = kOffCoarse + size_t(kCSites) * sizeof(float4) + 128;  // 86,272 B
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
  return lz * kSPlane + ly * kSX + ((lx & 1) ? kSHalf + (lx >> 1) : (lx >> 1));
}
__device__ __forceinline__ int rsite(int lx, int ly, int lz) { return lz * kSPlane + ly * kSX + lx; }

// Origin (x0, y0, z0) of tile b, tiles ordered x fastest so that neighbouring CTAs share halos.
__device__ __forceinline__ void tile_origin(const Dims& d, unsigned b, int& x0, int& y0, int& z0) {
  const unsigned ntx = unsigned(d.nx / kTX), nty = unsigned(d.ny / kTY);
  const unsigned q = b / ntx;
  x0 = int(b - q * ntx) * kTX;
  y0 = int(q % nty) * kTY;
  z0 = int(q / nty) * kTZ;
}

// ---- the right-hand-side copy: TMA tensor load completing on an mbarrier ----------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Thread 0 initialises the barrier and starts the copy of the tile's right-hand side; the barrier
// initialisation is published to the other threads by the __syncthreads() that precedes the wait.
__device__ __forceinline__ void tile_f_copy_start(const CUtensorMap* fmap, float* fsm, uint64_t* bar, int x0, int y0,
                                                  int z0) {
  if (threadIdx.x == 0) {
    const uint32_t b = smem_addr(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(b), "r"(1) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(kFBytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_addr(fsm)),
        "l"(reinterpret_cast<uint64_t>(fmap)), "r"(x0), "r"(y0), "r"(z0), "r"(0), "r"(b)
        : "memory");
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

// Bounded wait for the copy. Returns false in every thread of the CTA if any thread ran out of
// polls; then the solve is flagged (timeout + done) and the CTA waits once more, again bounded,
// for the copy it issued before it returns.
__device__ __forceinline__ bool tile_f_copy_wait(uint64_t* bar, SolveScalars* sc) {
  bool ok = false;
  for (int i = 0; i < kTileWaitPolls && !ok; i++) ok = mbar_try_wait(bar, 0);
  if (!__syncthreads_or(!ok)) return true;
  if (threadIdx.x == 0 && sc) {
    atomicExch(&sc->timeout, 1);
    atomicExch(&sc->done, 1);
  }
  for (int i = 0; i < kTileWaitPolls && !ok; i++) ok = mbar_try_wait(bar, 0);
  __syncthreads();
  return false;
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
// (lx, ly, lz0 .. lz0 + 3) of its column segment, reading planes lz0 - 1 .. lz0 + 4. fsm is the
// staged right-hand side (box order: x, y, z, case), fs the per-case scale applied to it.
template <int PX, int PY>
__device__ __forceinline__ void tile_pass(float4* sm, const float* fsm, const FineOp& op, const float (&fs)[3]) {
  const int t = int(threadIdx.x);
  const int i = t & 7, j = (t >> 3) & 7, seg = t >> 6;
  const int lx = 2 * i + 1 + PX, ly = 2 * j + 1 + PY, lz0 = 1 + kSeg * seg;
  // positions of the left / right neighbour columns relative to the own site: the parity of lx
  // is fixed by the pass, so they are compile-time offsets in the parity-split row
  constexpr int oL = PX ? kSHalf - 1 : -kSHalf, oR = PX ? kSHalf : -kSHalf + 1;
  const float* fcol = fsm + (ly - 1) * kTX + (lx - 1);
  float Kp[4] = {0.f, 0.f, 0.f, 0.f};  // conductivities of the previous plane
  PlaneCoef Cp;                        // coefficients of the previous plane
  float accA[3] = {0.f, 0.f, 0.f}, accB[3] = {0.f, 0.f, 0.f}, accC[3] = {0.f, 0.f, 0.f};  // P-1, P, P+1
  float dA = 0.f, dB = 0.f;  // their conductivity sums so far
#pragma unroll
  for (int s = 0; s < kSeg + 2; s++) {
    const int P = lz0 - 1 + s;
    const float4* b = sm + tsite(lx, ly, P);
    float4 nb[8];
    nb[0] = b[oL - kSX];
    nb[1] = b[-kSX];
    nb[2] = b[oR - kSX];
    nb[3] = b[oL];
    nb[4] = b[oR];
    nb[5] = b[oL + kSX];
    nb[6] = b[kSX];
    nb[7] = b[oR + kSX];
    const float kown = reinterpret_cast<const float*>(b)[3];
    const float K[4] = {nb[0].w, nb[1].w, nb[3].w, kown};
    const float sK = (K[0] + K[1]) + (K[2] + K[3]);
    PlaneCoef C;
    C.make(K, op);
    // vertex P + 1 (segment index s): its lower element plane is P
    float dC = 0.f;
    if (s < kSeg) {
      const float* fv = fcol + (lz0 - 1 + s) * (kTX * kTY);
#pragma unroll
      for (int c = 0; c < 3; c++) accC[c] = fv[c * (kTX * kTY * kTZ)] * fs[c];
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
      const size_t g = size_t(x0 + 4 * q) +
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
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int lx = 1 + 4 * q + e;
        float4 v = make_float4(0.f, 0.f, 0.f, kq[it][e]);
        if (kWithU) {
          v.x = uq[it][0][e];
          v.y = uq[it][1][e];
          v.z = uq[it][2][e];
          if (prolong) {
            const float3 p = prolong_site(cb, x0 + 4 * q + e, y0 - 1 + ly, z0 - 1 + lz, c0x, c0y, c0z);
            v.x += p.x;
            v.y += p.y;
            v.z += p.z;
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

// One smoothing leg of the fine level on a tile.
//   kPost = false (pre-smoothing): the leg starts from u = 0 (the halo stays 0), runs `sweeps`
//     sweeps in the pair order 0,1,2,3 and writes the interior to u_out.
//   kPost = true (post-smoothing): the tile is staged from u_in + P u_c (trilinear prolongation of
//     the coarse correction uc, homogenization/grid.cu:881-940), then `sweeps` sweeps in the order
//     3,2,1,0; the interior goes to u_out, which must not alias u_in.
// ks: fine conductivity (storage KT); fmap: TMA map of the right-hand side (FP32, 3 cases, scaled
// per case by fscale when given); u_in / u_out in storage VT; arithmetic and shared memory FP32.
template <bool kPost, typename KT, typename VT>
__global__ void __launch_bounds__(kSmoothThreads, 2)
    k_tile_smooth(const __grid_constant__ CUtensorMap fmap, Dims d, Dims dc, const KT* __restrict__ ks, FineOp op,
                  const VT* __restrict__ u_in, const float* __restrict__ uc, VT* __restrict__ u_out,
                  const double* fscale, int sweeps, SolveScalars* sc) {
  unsigned char* base = tile_smem_base();
  float* fsm = reinterpret_cast<float*>(base);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + kOffBar);
  float4* sm = reinterpret_cast<float4*>(base + kOffSites);
  float4* cb = reinterpret_cast<float4*>(base + kOffCoarse);
  pdl_wait();
  if (sc && solve_done(sc)) return;
  int x0, y0, z0;
  tile_origin(d, blockIdx.x, x0, y0, z0);
  const size_t nv = d.nv();
  tile_f_copy_start(&fmap, fsm, bar, x0, y0, z0);
  float fs[3] = {1.f, 1.f, 1.f};
  if (fscale)
#pragma unroll
    for (int c = 0; c < 3; c++) fs[c] = float(fscale[c]);
  stage_tile<kPost, kSmoothThreads, true>(d, dc, x0, y0, z0, ks, u_in, uc, sm, cb);
  __syncthreads();
  if (!tile_f_copy_wait(bar, sc)) return;
  for (int sw = 0; sw < sweeps; sw++) {
    if (!kPost) {
      tile_pass<0, 0>(sm, fsm, op, fs);
      __syncthreads();
      tile_pass<1, 0>(sm, fsm, op, fs);
      __syncthreads();
      tile_pass<0, 1>(sm, fsm, op, fs);
      __syncthreads();
      tile_pass<1, 1>(sm, fsm, op, fs);
      __syncthreads();
    } else {
      tile_pass<1, 1>(sm, fsm, op, fs);
      __syncthreads();
      tile_pass<0, 1>(sm, fsm, op, fs);
      __syncthreads();
      tile_pass<1, 0>(sm, fsm, op, fs);
      __syncthreads();
      tile_pass<0, 0>(sm, fsm, op, fs);
      __syncthreads();
    }
  }
  // interior back to global memory, 4 consecutive x at a time
  for (int w = int(threadIdx.x); w < kTX * kTY * kTZ / 4; w += kSmoothThreads) {
    const int q = w & 3, row = w >> 2;
    const int ly = 1 + row % kTY, lz = 1 + row / kTY;
    float o0[4], o1[4], o2[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
      const float4 v = sm[tsite(1 + 4 * q + e, ly, lz)];
      o0[e] = v.x, o1[e] = v.y, o2[e] = v.z;
    }
    const size_t g = size_t(x0 + 4 * q) + size_t(d.nx) * (size_t(y0 + ly - 1) + size_t(d.ny) * size_t(z0 + lz - 1));
    st4(u_out + g, o0);
    st4(u_out + nv + g, o1);
    st4(u_out + 2 * nv + g, o2);
  }
}

// r = f - A u on the fine level for every vertex of a tile, from a staged tile with its halo
// (natural site order here: lanes take consecutive sites of a row). A thread owns one column of
// the tile and streams its 10 planes.
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
  tile_origin(d, blockIdx.x, x0, y0, z0);
  const size_t nv = d.nv();
  tile_f_copy_start(&fmap, fsm, bar, x0, y0, z0);
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
  const float* fcol = fsm + (ly - 1) * kTX + (lx - 1);
  float Kp[4] = {0.f, 0.f, 0.f, 0.f};
  PlaneCoef Cp;
  float accA[3] = {0.f, 0.f, 0.f}, accB[3] = {0.f, 0.f, 0.f}, accC[3] = {0.f, 0.f, 0.f};
  float dA = 0.f, dB = 0.f;
  float uA[3] = {0.f, 0.f, 0.f}, uB[3] = {0.f, 0.f, 0.f};  // own values of the vertices P - 1, P
#pragma unroll 1
  for (int P = 0; P < kSZ; P++) {
    const float4* b = sm + rsite(lx, ly, P);
    float4 nb[8];
    nb[0] = b[-kSX - 1];
    nb[1] = b[-kSX];
    nb[2] = b[-kSX + 1];
    nb[3] = b[-1];
    nb[4] = b[1];
    nb[5] = b[kSX - 1];
    nb[6] = b[kSX];
    nb[7] = b[kSX + 1];
    const float4 own = b[0];
    const float K[4] = {nb[0].w, nb[1].w, nb[3].w, own.w};
    const float sK = (K[0] + K[1]) + (K[2] + K[3]);
    PlaneCoef C;
    C.make(K, op);
    float dC = 0.f;
    // vertex P + 1 (interior planes 1..8): lower element plane P
    if (P + 1 <= kTZ) {
      const float* fv = fcol + P * (kTX * kTY);
#pragma unroll
      for (int c = 0; c < 3; c++) accC[c] = fv[c * (kTX * kTY * kTZ)] * fs[c];
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

}  // namespace otm
