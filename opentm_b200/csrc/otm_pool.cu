// otm_pool.cu -- stream-ordered scratch memory of the handle-free entry points.
//
// The OC update, the OC sensitivity filter, the MMA subsolver and the server's task tables need
// temporary device buffers per call. They take them from one memory pool per device owned by
// the library, whose release threshold keeps freed memory cached: after the first calls every
// allocation is served from the pool without a driver call, and synchronising a stream never
// hands the memory back to the driver (the device's default pool would, and the next call would
// then pay for a fresh allocation).
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <mutex>

#include "otm_common.cuh"

namespace otm {

namespace {
constexpr int kPoolMaxDevices = 64;
cudaMemPool_t g_pools[kPoolMaxDevices] = {};
std::mutex g_pool_mu;
std::atomic<uint64_t> g_scratch_allocs{0};
}  // namespace

cudaError_t scratch_malloc(void** p, size_t bytes, cudaStream_t s) {
  g_scratch_allocs.fetch_add(1, std::memory_order_relaxed);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kPoolMaxDevices) return cudaErrorInvalidDevice;
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (!g_pools[dev]) {
      cudaMemPoolProps props{};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      e = cudaMemPoolCreate(&g_pools[dev], &props);
      if (e != cudaSuccess) {
        g_pools[dev] = nullptr;
        return e;
      }
      uint64_t keep = UINT64_MAX;
      e = cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) return e;
    }
    pool = g_pools[dev];
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

}  // namespace otm

extern "C" {

uint64_t otm_scratch_alloc_count(void) { return otm::g_scratch_allocs.load(); }

otm_status otm_host_alloc(size_t bytes, void** out) {
  if (!out || bytes == 0) return OTM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const cudaError_t e = cudaHostAlloc(out, bytes, cudaHostAllocPortable);
  if (e != cudaSuccess) {
    *out = nullptr;
    return otm::cuda_fail(e, "cudaHostAlloc");
  }
  return OTM_OK;
}

otm_status otm_copy_to_device(void* dst_dev, const void* src_host, size_t bytes, void* stream) {
  if ((!dst_dev || !src_host) && bytes) return OTM_ERR_INVALID_ARGUMENT;
  if (!bytes) return OTM_OK;
  const cudaError_t e = cudaMemcpyAsync(dst_dev, src_host, bytes, cudaMemcpyHostToDevice, (cudaStream_t)stream);
  return e == cudaSuccess ? OTM_OK : otm::cuda_fail(e, "otm_copy_to_device");
}

otm_status otm_copy_to_host(void* dst_host, const void* src_dev, size_t bytes, void* stream) {
  if ((!dst_host || !src_dev) && bytes) return OTM_ERR_INVALID_ARGUMENT;
  if (!bytes) return OTM_OK;
  const cudaError_t e = cudaMemcpyAsync(dst_host, src_dev, bytes, cudaMemcpyDeviceToHost, (cudaStream_t)stream);
  return e == cudaSuccess ? OTM_OK : otm::cuda_fail(e, "otm_copy_to_host");
}

otm_status otm_host_free(void* p) {
  if (!p) return OTM_OK;
  const cudaError_t e = cudaFreeHost(p);
  return e == cudaSuccess ? OTM_OK : otm::cuda_fail(e, "cudaFreeHost");
}

}  // extern "C"
