// otm_common.cuh -- shared host/device helpers of the B200 homogenization library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "opentm_b200.h"

namespace otm {

// Conductivity floor added inside the solver (homogenization/grid.h:429).
constexpr float kRhoPenalMin = 1e-9f;

// Block size of the stencil kernels and reductions.
constexpr int kBlock = 256;
// Fixed upper bound on reduction partial slots per launch (deterministic ordering).
constexpr int kMaxPartials = 2048;

// Process-wide count of kernel launches issued by the library.
void count_launches(uint64_t n);

// Per-thread message of the last failure, returned by otm_last_error().
void set_error(const std::string& msg);
otm_status cuda_fail(cudaError_t e, const char* what);
// Stream-ordered scratch from the library's per-device memory pool (freed with cudaFreeAsync).
cudaError_t scratch_malloc(void** p, size_t bytes, cudaStream_t s);

#define OTM_CUDA(call)                                  \
  do {                                                  \
    cudaError_t e__ = (call);                           \
    if (e__ != cudaSuccess) return ::otm::cuda_fail(e__, #call); \
  } while (0)

#define OTM_CHECK_LAUNCH(what)                          \
  do {                                                  \
    cudaError_t e__ = cudaGetLastError();               \
    if (e__ != cudaSuccess) return ::otm::cuda_fail(e__, what); \
  } while (0)

#define OTM_TRY(expr)                                   \
  do {                                                  \
    otm_status s__ = (expr);                            \
    if (s__ != OTM_OK) return s__;                      \
  } while (0)

// Periodic grid dimensions, x fastest: id = x + nx (y + ny z).
struct Dims {
  int nx, ny, nz;
  __host__ __device__ size_t nv() const { return size_t(nx) * ny * nz; }
};

// Programmatic dependent launch: waits until the grids this launch depends on have completed
// and their memory is visible. A kernel launched with the programmatic-serialization attribute
// may start while its predecessor drains, so this must come before any read of data that the
// predecessor writes; for a launch without the attribute it returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// This CTA's share of an L2 prefetch of [base, base + bytes) (base 16-byte aligned, or null for
// none), issued by thread 0 as bulk prefetches of at most 32 KB (cp.async.bulk.prefetch.L2: a
// hint that moves the lines into L2 through the copy engine and holds no registers or shared
// memory). Used by a kernel to bring the data of the kernel after it into L2 while it runs.
__device__ __forceinline__ void l2_prefetch_share(const void* base, size_t bytes) {
  if (base == nullptr || threadIdx.x != 0) return;
  const size_t per = ((bytes + gridDim.x - 1) / gridDim.x + 15) & ~size_t(15);
  size_t lo = size_t(blockIdx.x) * per;
  const size_t hi = lo + per < bytes ? lo + per : bytes;
  for (; lo + 16 <= hi; lo += 32768) {
    const size_t rest = hi - lo;
    const unsigned n = unsigned(rest < 32768 ? rest : 32768) & ~15u;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(static_cast<const char*>(base) + lo), "r"(n)
                 : "memory");
  }
}

// (x, y, z) of lexicographic index v (x fastest) on a grid with rows of nx and planes of
// nx * ny points. Grids hold at most 1024^3 = 2^30 points, so 32-bit division is exact and
// several times cheaper than 64-bit.
struct Coord3 {
  int x, y, z;
};
__host__ __device__ __forceinline__ Coord3 split3(size_t v, int nx, int ny) {
  const unsigned u = unsigned(v), unx = unsigned(nx), uny = unsigned(ny);
  const unsigned q = u / unx;
  return Coord3{int(u - q * unx), int(q % uny), int(q / uny)};
}

__device__ __forceinline__ int wrapm(int a, int n) {
  // a in [-n, 2n)
  return a < 0 ? a + n : (a >= n ? a - n : a);
}

// Deterministic FP64 block reduction of NV values per thread (warp shuffles then shared
// memory, fixed order). The result is valid in thread 0 only.
template <int NV>
__device__ __forceinline__ void block_reduce_f64(double (&v)[NV], double* smem /* >= 32*NV */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < NV; i++) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[i] += __shfl_down_sync(0xffffffffu, v[i], off);
  }
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) smem[warp * NV + i] = v[i];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < NV; i++) {
      double x = lane < nwarps ? smem[lane * NV + i] : 0.0;
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
      v[i] = x;
    }
  }
}

inline int ceil_div(size_t a, size_t b) { return int((a + b - 1) / b); }

}  // namespace otm
