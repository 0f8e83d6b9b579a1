// otm_oc.cu -- OCOptimizer on the device (optimization/OCOptimizer.cu:12-152).
//
// The reference runs 20 host-driven bisection steps, each one kernel, one FP32 reduction and
// one device-to-host copy. Here the whole bisection is a fixed sequence of kernels that keep
// the multiplier bracket on the device (last-block finalisation, FP64 volume sums), so the
// host never waits; a converged bisection turns the remaining steps into no-ops.
#include <cuda_runtime.h>

#include <cmath>

#include "otm_common.cuh"
#include "otm_mg_kernels.cuh"

namespace otm {

struct OcState {
  double gmax, gmin, g, vol;
  int done;
  int iters;
  unsigned int counter;
  int pad;
};

constexpr int kOcSteps = 20;  // OCOptimizer.cu:69

// Move limit and box bounds of the OC update, in the reference's order.
__device__ __forceinline__ float oc_clamp(float nr, float r, float min_rho, float step) {
  if (nr - r < -step) nr = r - step;
  if (nr - r > step) nr = r + step;
  if (nr < min_rho) nr = min_rho;
  if (nr > 1.f) nr = 1.f;
  return nr;
}

// rho_new = clamp(r * (-s/g)^damp) (optimization/OCOptimizer.cu:12-39), FP32 as the reference.
__device__ __forceinline__ float oc_new_rho(float s, float r, float g, float min_rho, float step, float damp) {
  float B = -s / g;
  if (B < 0.f) B = 0.01f;
  const float nr = (damp == 0.5f ? sqrtf(B) : powf(B, damp)) * r;
  return oc_clamp(nr, r, min_rho, step);
}

__global__ void __launch_bounds__(kBlock) k_oc_maxabs(int ne, const float* __restrict__ sens, double* partials,
                                                      OcState* st) {
  __shared__ double smem[32];
  double m = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += gridDim.x * blockDim.x)
    m = fmax(m, fabs(double(sens[i])));
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
  if ((threadIdx.x & 31) == 0) smem[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < (blockDim.x + 31) / 32; w++) b = fmax(b, smem[w]);
    partials[blockIdx.x] = b;
  }
  if (last_block(&st->counter)) {
    double b = 0.0;
#pragma unroll 4
    for (int i = threadIdx.x; i < int(gridDim.x); i += blockDim.x) b = fmax(b, __ldcg(partials + i));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) b = fmax(b, __shfl_down_sync(0xffffffffu, b, off));
    __syncthreads();
    if ((threadIdx.x & 31) == 0) smem[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 0; w < (blockDim.x + 31) / 32; w++) b = fmax(b, smem[w]);
      st->gmax = b;
      st->gmin = 0.0;
      st->g = b / 2;
      st->done = 0;
      st->iters = 0;
      st->counter = 0;
    }
  }
}

// Five bisection steps per pass: the volumes of all 31 multipliers the bisection can visit
// in its next 5 steps (the nodes of the bisection tree below [gmin, gmax], midpoints in FP32
// as the reference computes them) are summed in one read of sens and rho; the last block
// then walks the tree exactly as the sequential loop would (OCOptimizer.cu:69-88).
constexpr int kTreeDepth = 5;
constexpr int kTreeNodes = (1 << kTreeDepth) - 1;

// Node i of the bisection tree below [gmin, gmax]: midpoints in FP32, children 2i+1 (volume
// too small: gmax = g) and 2i+2 (volume too large: gmin = g).
__device__ void oc_tree(float gmin, float gmax, float* g) {
  float lo[kTreeNodes], hi[kTreeNodes];
  lo[0] = gmin;
  hi[0] = gmax;
  for (int i = 0; i < kTreeNodes; i++) {
    g[i] = (hi[i] + lo[i]) / 2;
    if (2 * i + 2 < kTreeNodes) {
      lo[2 * i + 1] = lo[i];
      hi[2 * i + 1] = g[i];
      lo[2 * i + 2] = g[i];
      hi[2 * i + 2] = hi[i];
    }
  }
}

__global__ void __launch_bounds__(kBlock) k_oc_tree_pass(int ne, const float* __restrict__ sens,
                                                         const float* __restrict__ rho, float volratio, float min_rho,
                                                         float step, float damp, double* partials, OcState* st) {
  if (*((volatile int*)&st->done)) return;
  __shared__ float g[kTreeNodes];
  __shared__ float cf[kTreeNodes];
  __shared__ float wsum[kBlock / 32][kTreeNodes];
  if (threadIdx.x == 0) oc_tree(float(st->gmin), float(st->gmax), g);
  __syncthreads();
  // (-s/g)^damp = (-s)^damp * g^-damp for s < 0: the candidate factor g^-damp is computed once
  // per block and the element factor once per element, so a candidate costs one multiply and
  // the clamps instead of a division and a square root. The volumes only steer the bisection;
  // the new densities themselves (k_oc_apply) use the reference's expression.
  if (threadIdx.x < kTreeNodes)
    cf[threadIdx.x] = damp == 0.5f ? float(1.0 / sqrt(double(g[threadIdx.x])))
                                    : float(pow(double(g[threadIdx.x]), -double(damp)));
  __syncthreads();
  // per-thread FP32 partial volumes of the 31 candidates (a few elements per thread); the
  // candidate factors live in registers, and the move limit and box bounds are one interval
  // [max(r - step, min_rho), min(r + step, 1)] (the same clamp for min_rho <= r <= 1)
  float v[kTreeNodes], cfr[kTreeNodes];
#pragma unroll
  for (int t = 0; t < kTreeNodes; t++) {
    v[t] = 0.f;
    cfr[t] = cf[t];
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += gridDim.x * blockDim.x) {
    const float s = __ldg(sens + i), r = __ldg(rho + i);
    if (s < 0.f) {
      const float a = (damp == 0.5f ? sqrtf(-s) : powf(-s, damp)) * r;
      const float lo = fmaxf(r - step, min_rho), hi = fminf(r + step, 1.f);
#pragma unroll
      for (int t = 0; t < kTreeNodes; t++) v[t] += fminf(fmaxf(a * cfr[t], lo), hi);
    } else {  // -s/g <= 0 (or NaN): the same value for every candidate
      const float nr = oc_new_rho(s, r, g[0], min_rho, step, damp);
#pragma unroll
      for (int t = 0; t < kTreeNodes; t++) v[t] += nr;
    }
  }
#pragma unroll
  for (int t = 0; t < kTreeNodes; t++)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v[t] += __shfl_down_sync(0xffffffffu, v[t], off);
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int t = 0; t < kTreeNodes; t++) wsum[threadIdx.x >> 5][t] = v[t];
  __syncthreads();
  if (threadIdx.x < kTreeNodes) {
    double b = 0.0;
    for (int w = 0; w < int(blockDim.x) / 32; w++) b += double(wsum[w][threadIdx.x]);
    partials[threadIdx.x * gridDim.x + blockIdx.x] = b;  // candidate-major
  }
  if (last_block(&st->counter)) {
    // one warp per candidate sums the blocks' partials (coalesced, fixed order)
    __shared__ double tot[kTreeNodes];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = warp; t < kTreeNodes; t += int(blockDim.x >> 5)) {
      double a = 0.0;
      const double* col = partials + size_t(t) * gridDim.x;
#pragma unroll 8
      for (int b = lane; b < int(gridDim.x); b += 32) a += __ldcg(col + b);  // L2: never a stale L1 line
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
      if (lane == 0) tot[t] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int node = 0;
      for (int depth = 0; depth < kTreeDepth && !st->done; depth++) {
        const double vol = tot[node] / ne;
        st->vol = vol;
        st->g = double(g[node]);
        st->iters += 1;
        if (vol < volratio - 0.0001) {
          st->gmax = double(g[node]);
          node = 2 * node + 1;
        } else if (vol > volratio + 0.0001) {
          st->gmin = double(g[node]);
          node = 2 * node + 2;
        } else {
          st->done = 1;
        }
        if (st->iters >= kOcSteps) st->done = 1;
      }
      st->counter = 0;
    }
  }
}

// One bisection step: volume of the candidate density at g = (gmax + gmin) / 2.
__global__ void __launch_bounds__(kBlock) k_oc_pass(int ne, const float* __restrict__ sens,
                                                    const float* __restrict__ rho, float volratio, float min_rho,
                                                    float step, float damp, double* partials, OcState* st) {
  if (*((volatile int*)&st->done)) return;
  __shared__ double smem[32];
  const float g = float((st->gmax + st->gmin) / 2);
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ne; i += gridDim.x * blockDim.x)
    v[0] += oc_new_rho(__ldg(sens + i), __ldg(rho + i), g, min_rho, step, damp);
  block_reduce_f64<1>(v, smem);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
  if (last_block(&st->counter)) {
    double t[1];
    reduce_partials<1>(partials, gridDim.x, t, smem);
    if (threadIdx.x == 0) {
      const double vol = t[0] / ne;
      st->vol = vol;
      st->g = double(g);
      st->iters += 1;
      if (vol < volratio - 0.0001)
        st->gmax = double(g);
      else if (vol > volratio + 0.0001)
        st->gmin = double(g);
      else
        st->done = 1;
      if (st->iters >= kOcSteps) st->done = 1;
      st->counter = 0;
    }
  }
}

__global__ void __launch_bounds__(kBlock) k_oc_apply(int ne, const float* __restrict__ sens, float* rho,
                                                     float min_rho, float step, float damp, const OcState* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  rho[i] = oc_new_rho(sens[i], rho[i], float(st->g), min_rho, step, damp);
}

// Sensitivity filter: periodic Linear weights, s_e <- sum w s rho / (sum w * rho_e).
struct OcFilterWeights {
  int half, taps;
  float w[13 * 13 * 13];
};

__global__ void __launch_bounds__(256) k_oc_filter(Dims d, const float* __restrict__ sens,
                                                   const float* __restrict__ rho, size_t pitch, float* __restrict__ out,
                                                   OcFilterWeights fw) {
  const size_t nv = d.nv();
  const size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const Coord3 c3_ = split3(v, d.nx, d.ny);
    const int x = c3_.x, y = c3_.y, z = c3_.z;
  const int h = fw.half, w1 = 2 * h + 1;
  float sum = 0.f, ws = 0.f;
  for (int t = 0; t < fw.taps; t++) {
    const int ox = t % w1 - h, oy = (t / w1) % w1 - h, oz = t / (w1 * w1) - h;
    const int px = ((x + ox) % d.nx + d.nx) % d.nx, py = ((y + oy) % d.ny + d.ny) % d.ny,
              pz = ((z + oz) % d.nz + d.nz) % d.nz;
    const size_t q = (size_t(py) + size_t(d.ny) * pz) * pitch + px;
    const float w = fw.w[t];
    sum += __ldg(sens + q) * __ldg(rho + q) * w;
    ws += w;
  }
  const size_t e = (size_t(y) + size_t(d.ny) * z) * pitch + x;
  out[v] = sum / (ws * __ldg(rho + e));
}

__global__ void __launch_bounds__(256) k_copy_pitched(Dims d, const float* __restrict__ src, float* dst,
                                                      size_t pitch) {
  const size_t nv = d.nv();
  const size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const int x = int(v % d.nx);
  dst[(v / d.nx) * pitch + x] = src[v];
}

}  // namespace otm

using namespace otm;

extern "C" {

otm_status otm_oc_filter_sens(float* sens, const float* rho, size_t pitchT, const int reso[3], float radius,
                              void* stream) {
  if (!sens || !rho || !reso || reso[0] < 1 || reso[1] < 1 || reso[2] < 1) return OTM_ERR_INVALID_ARGUMENT;
  const Dims d{reso[0], reso[1], reso[2]};
  if (pitchT == 0) pitchT = size_t(d.nx);
  if (pitchT < size_t(d.nx)) return OTM_ERR_INVALID_ARGUMENT;
  const int h = int(radius + 0.5f);
  if (!(radius > 0.f) || h > 6) {
    set_error("filter radius must be in (0, 6.5)");
    return OTM_ERR_INVALID_ARGUMENT;
  }
  OcFilterWeights fw;
  fw.half = h;
  fw.taps = (2 * h + 1) * (2 * h + 1) * (2 * h + 1);
  float wsum = 0.f;
  for (int t = 0; t < fw.taps; t++) {
    const int ox = t % (2 * h + 1) - h, oy = t / (2 * h + 1) % (2 * h + 1) - h, oz = t / ((2 * h + 1) * (2 * h + 1)) - h;
    const float q2 = float(ox * ox + oy * oy + oz * oz) / (radius * radius);
    fw.w[t] = q2 < 1.f ? 1.f - std::sqrt(q2) : 0.f;  // WeightFunc<Linear>
    wsum += fw.w[t];
  }
  for (int t = 0; t < fw.taps; t++) fw.w[t] /= wsum;
  cudaStream_t s = (cudaStream_t)stream;
  float* tmp = nullptr;
  OTM_CUDA(scratch_malloc((void**)&tmp, d.nv() * sizeof(float), s));
  k_oc_filter<<<ceil_div(d.nv(), 256), 256, 0, s>>>(d, sens, rho, pitchT, tmp, fw);
  k_copy_pitched<<<ceil_div(d.nv(), 256), 256, 0, s>>>(d, tmp, sens, pitchT);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(tmp, s);
  if (e != cudaSuccess) return cuda_fail(e, "k_oc_filter");
  count_launches(2);
  return OTM_OK;
}

otm_status otm_oc_update(int ne, const float* sens, float* rho, float volratio, float min_rho, float step_limit,
                         float damp, void* stream, int* iters_out) {
  if (ne <= 0 || !sens || !rho) return OTM_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  const int nb = std::min(kMaxPartials, std::max(1, (ne + kBlock - 1) / kBlock));
  char* scratch = nullptr;
  const size_t bytes = sizeof(OcState) + size_t(nb) * kTreeNodes * sizeof(double);
  OTM_CUDA(scratch_malloc((void**)&scratch, bytes, s));
  OcState* st = (OcState*)scratch;
  double* partials = (double*)(scratch + sizeof(OcState));
  cudaMemsetAsync(st, 0, sizeof(OcState), s);
  k_oc_maxabs<<<nb, kBlock, 0, s>>>(ne, sens, partials, st);
  // the tree passes run two blocks per SM: a thread then sums a few dozen elements before its
  // 31 candidate sums are reduced, instead of the reduction costing as much as its elements
  // (one pass at 128^3: 38.8 / 26.9 / 32.0 / 39.0 us with 1 / 2 / 4 / 8 blocks per SM)
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    sms = 148;
  const int nbt = std::min(nb, 2 * sms);
  for (int i = 0; i < (kOcSteps + kTreeDepth - 1) / kTreeDepth; i++)
    k_oc_tree_pass<<<nbt, kBlock, 0, s>>>(ne, sens, rho, volratio, min_rho, step_limit, damp, partials, st);
  k_oc_apply<<<ceil_div(size_t(ne), kBlock), kBlock, 0, s>>>(ne, sens, rho, min_rho, step_limit, damp, st);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess && iters_out) {
    OcState h;
    e = cudaMemcpyAsync(&h, st, sizeof(OcState), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    *iters_out = h.iters;
  }
  cudaFreeAsync(scratch, s);
  if (e != cudaSuccess) return cuda_fail(e, "otm_oc_update");
  count_launches(2 + (kOcSteps + kTreeDepth - 1) / kTreeDepth);
  return OTM_OK;
}

}  // extern "C"
