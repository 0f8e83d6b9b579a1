// otm_noalloc.cu -- the OC sensitivity filter without any device allocation.
//
// For callers that cannot allocate GPU memory while they run (their allocator already owns the
// device's memory, or a cudaMalloc/cudaFree with its possible device-wide synchronisation is
// not allowed in their loop). The filter's temporary copy lives in `g_noalloc_scratch`, a
// file-scope device array of OTM_NOALLOC_MAX_CELLS floats that every GPU loading the library
// holds until the process exits. In host code that symbol is only a host-side stand-in, never
// a device address: its device address is looked up once per device with
// cudaGetSymbolAddress while that device is current, and that pointer is what the kernels
// get. Calls share the array, so calls whose GPU work overlaps race on it.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "opentm_b200_noalloc.h"
#include "otm_common.cuh"

namespace otm {

static __device__ __align__(256) float g_noalloc_scratch[OTM_NOALLOC_MAX_CELLS];

constexpr int kNaMaxDevices = 64;
static float* g_scratch_ptr[kNaMaxDevices] = {};
static std::mutex g_scratch_mu;

// Device address of the scratch array on the current device (looked up on first use).
static otm_status scratch_address(float** out) {
  int dev = 0;
  OTM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNaMaxDevices) {
    set_error("device ordinal out of range for the allocation-free filter");
    return OTM_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_scratch_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_scratch_ptr[dev];
  return OTM_OK;
}

constexpr int kNaMaxHalf = 6;

struct NaWeights {
  int half, taps;
  float w[(2 * kNaMaxHalf + 1) * (2 * kNaMaxHalf + 1) * (2 * kNaMaxHalf + 1)];
};

// s_new(e) = sum_n w s_n rho_n / (sum_n w * rho_e) over the periodic Linear neighbourhood
// (optimization/OCOptimizer.cu:76-104), written unpitched into the scratch array.
static __global__ void __launch_bounds__(256) k_filter_to_scratch(Dims d, const float* __restrict__ sens,
                                                                  const float* __restrict__ rho, size_t pitch,
                                                                  float* __restrict__ scratch, NaWeights fw) {
  const size_t nv = d.nv();
  const size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const int x = int(v % d.nx), y = int((v / d.nx) % d.ny), z = int(v / (size_t(d.nx) * d.ny));
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
  scratch[v] = sum / (ws * __ldg(rho + e));
}

static __global__ void __launch_bounds__(256) k_scratch_to_sens(Dims d, const float* __restrict__ scratch, float* sens,
                                                                size_t pitch) {
  const size_t nv = d.nv();
  const size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  sens[(v / d.nx) * pitch + v % d.nx] = scratch[v];
}

}  // namespace otm

using namespace otm;

extern "C" otm_status otm_oc_filter_sens_noalloc(float* sens, const float* rho, size_t pitchT, const int reso[3],
                                                 float radius, void* stream) {
  if (!sens || !rho || !reso || reso[0] < 1 || reso[1] < 1 || reso[2] < 1) return OTM_ERR_INVALID_ARGUMENT;
  const Dims d{reso[0], reso[1], reso[2]};
  if (d.nv() > size_t(OTM_NOALLOC_MAX_CELLS)) {
    set_error("the allocation-free filter accepts at most OTM_NOALLOC_MAX_CELLS (2^21 = 128^3) voxels");
    return OTM_ERR_UNSUPPORTED;
  }
  if (pitchT == 0) pitchT = size_t(d.nx);
  if (pitchT < size_t(d.nx)) return OTM_ERR_INVALID_ARGUMENT;
  const int h = int(radius + 0.5f);
  if (!(radius > 0.f) || h > kNaMaxHalf) {
    set_error("filter radius must be in (0, 6.5)");
    return OTM_ERR_INVALID_ARGUMENT;
  }
  NaWeights fw;
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
  float* scratch = nullptr;
  OTM_TRY(scratch_address(&scratch));
  cudaStream_t s = (cudaStream_t)stream;
  k_filter_to_scratch<<<ceil_div(d.nv(), 256), 256, 0, s>>>(d, sens, rho, pitchT, scratch, fw);
  k_scratch_to_sens<<<ceil_div(d.nv(), 256), 256, 0, s>>>(d, scratch, sens, pitchT);
  OTM_CHECK_LAUNCH("otm_oc_filter_sens_noalloc");
  count_launches(2);
  return OTM_OK;
}
