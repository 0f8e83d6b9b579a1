// otm_filter.cu -- density filter (radial convolution with in-bounds renormalisation), the
// fused SIMP density chain and their adjoints (AutoDiff/TensorExpression.h:993-1185,
// AutoDiff/TensorExpression.cuh:281-385).
//
// One thread per voxel; the (2h+1)^3 normalised weights travel as a kernel parameter
// (constant bank, broadcast to the warp), so no device allocation or global state is used.
#include <cuda_runtime.h>

#include <cmath>

#include "otm_common.cuh"

namespace otm {

constexpr int kMaxHalf = 6;
constexpr int kMaxTaps = (2 * kMaxHalf + 1) * (2 * kMaxHalf + 1) * (2 * kMaxHalf + 1);

struct ConvWeights {
  int half;  // h = int(radius + 0.5)
  int taps;  // (2h+1)^3
  float w[kMaxTaps];  // w(off) / sum_cube w, off enumerated x fastest from -h
};

// Radial weight functions WeightFunc<Spline4> / WeightFunc<Linear>
// (AutoDiff/TensorExpression.h:1054-1077), evaluated in FP32 as in the reference.
static float radial_weight(int type, float r, int ox, int oy, int oz) {
  const float q2 = float(ox * ox + oy * oy + oz * oz) / (r * r);
  const float q = std::sqrt(q2);
  if (!(q2 < 1.f)) return 0.f;
  if (type == OTM_WEIGHT_SPLINE4) return 1.f - 6.f * q2 + 8.f * q2 * q - 3.f * q2 * q2;
  return 1.f - q;
}

static otm_status make_weights(int type, float radius, ConvWeights* cw) {
  if (type != OTM_WEIGHT_SPLINE4 && type != OTM_WEIGHT_LINEAR) {
    set_error("unknown filter weight type");
    return OTM_ERR_INVALID_ARGUMENT;
  }
  if (!(radius > 0.f)) {
    set_error("filter radius must be positive");
    return OTM_ERR_INVALID_ARGUMENT;
  }
  const int h = int(radius + 0.5f);  // convker_t halfdomain = r + 0.5 truncated (TensorExpression.h:1079-1093)
  if (h > kMaxHalf) {
    set_error("filter radius too large (half width must be <= 6)");
    return OTM_ERR_UNSUPPORTED;
  }
  cw->half = h;
  cw->taps = (2 * h + 1) * (2 * h + 1) * (2 * h + 1);
  float wsum = 0.f;
  for (int i = 0; i < cw->taps; i++) {
    const int ox = i % (2 * h + 1) - h, oy = i / (2 * h + 1) % (2 * h + 1) - h, oz = i / ((2 * h + 1) * (2 * h + 1)) - h;
    cw->w[i] = radial_weight(type, radius, ox, oy, oz);
    wsum += cw->w[i];
  }
  for (int i = 0; i < cw->taps; i++) cw->w[i] /= wsum;  // normalize = true
  return OTM_OK;
}

// Forward: out = sum_valid w src / sum_valid w; with fuse_simp it also writes
// k = (k0 - kmin) out^p + kmin and dk = dk/dout.
template <bool kSimp>
__global__ void __launch_bounds__(256) k_conv_forward(Dims d, const float* __restrict__ src, int src_pitch,
                                                      float* __restrict__ dst, int dst_pitch, float* __restrict__ wsum,
                                                      int periodic, ConvWeights cw, float p, float k0, float kmin,
                                                      float* __restrict__ kout, float* __restrict__ dkout) {
  const size_t nv = d.nv();
  const size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const int x = int(v % d.nx), y = int((v / d.nx) % d.ny), z = int(v / (size_t(d.nx) * d.ny));
  const int h = cw.half, w1 = 2 * h + 1;
  float sum = 0.f, ws = 0.f;
  for (int t = 0; t < cw.taps; t++) {
    const int ox = t % w1 - h, oy = (t / w1) % w1 - h, oz = t / (w1 * w1) - h;
    int px = x + ox, py = y + oy, pz = z + oz;
    const bool in = px >= 0 && px < d.nx && py >= 0 && py < d.ny && pz >= 0 && pz < d.nz;
    if (!in) {
      if (!periodic) continue;  // zero padding contributes nothing and no weight
      px = ((px % d.nx) + d.nx) % d.nx;
      py = ((py % d.ny) + d.ny) % d.ny;
      pz = ((pz % d.nz) + d.nz) % d.nz;
    }
    const float w = cw.w[t];
    sum += w * __ldg(src + (size_t(py) + size_t(d.ny) * pz) * src_pitch + px);
    ws += w;
  }
  const float out = sum / ws;
  const size_t o = (size_t(y) + size_t(d.ny) * z) * dst_pitch + x;
  if (dst) dst[o] = out;
  if (wsum) wsum[v] = ws;
  if (kSimp) {
    const float pw = (p == 3.f) ? out * out * out : powf(out, p);
    kout[v] = (k0 - kmin) * pw + kmin;
    const float dpw = (p == 3.f) ? 3.f * out * out : p * powf(out, p - 1.f);
    dkout[v] = (k0 - kmin) * dpw;
  }
}

// Adjoint: g_src(i) = sum_off w(off) g(i - off) / ws(i - off); with kChain the incoming
// gradient is g_k * dk (chain rule through the SIMP map, unarymap_backward).
template <bool kChain>
__global__ void __launch_bounds__(256) k_conv_backward(Dims d, const float* __restrict__ g, int g_pitch,
                                                       const float* __restrict__ dk, const float* __restrict__ wsum,
                                                       float* __restrict__ out, int out_pitch, int periodic,
                                                       ConvWeights cw) {
  const size_t nv = d.nv();
  const size_t v = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (v >= nv) return;
  const int x = int(v % d.nx), y = int((v / d.nx) % d.ny), z = int(v / (size_t(d.nx) * d.ny));
  const int h = cw.half, w1 = 2 * h + 1;
  float sum = 0.f;
  for (int t = 0; t < cw.taps; t++) {
    const int ox = t % w1 - h, oy = (t / w1) % w1 - h, oz = t / (w1 * w1) - h;
    int px = x - ox, py = y - oy, pz = z - oz;
    const bool in = px >= 0 && px < d.nx && py >= 0 && py < d.ny && pz >= 0 && pz < d.nz;
    if (!in) {
      if (!periodic) continue;
      px = ((px % d.nx) + d.nx) % d.nx;
      py = ((py % d.ny) + d.ny) % d.ny;
      pz = ((pz % d.nz) + d.nz) % d.nz;
    }
    const size_t q = (size_t(py) + size_t(d.ny) * pz) * d.nx + px;
    float gq = __ldg(g + (size_t(py) + size_t(d.ny) * pz) * g_pitch + px);
    if (kChain) gq *= __ldg(dk + q);
    sum += cw.w[t] * gq / __ldg(wsum + q);
  }
  out[(size_t(y) + size_t(d.ny) * z) * out_pitch + x] = sum;
}

static otm_status check_reso(const int reso[3]) {
  if (!reso || reso[0] < 1 || reso[1] < 1 || reso[2] < 1) {
    set_error("invalid resolution");
    return OTM_ERR_INVALID_ARGUMENT;
  }
  return OTM_OK;
}

}  // namespace otm

using namespace otm;

extern "C" {

otm_status otm_filter_forward(const int reso[3], const float* src, int src_pitchT, float* dst, int dst_pitchT,
                              float* wsum, int weight_type, float radius, int periodic, void* stream) {
  OTM_TRY(check_reso(reso));
  if (!src || !dst) return OTM_ERR_INVALID_ARGUMENT;
  const Dims d{reso[0], reso[1], reso[2]};
  if (src_pitchT <= 0) src_pitchT = d.nx;
  if (dst_pitchT <= 0) dst_pitchT = d.nx;
  if (src_pitchT < d.nx || dst_pitchT < d.nx) return OTM_ERR_INVALID_ARGUMENT;
  ConvWeights cw;
  OTM_TRY(make_weights(weight_type, radius, &cw));
  k_conv_forward<false><<<ceil_div(d.nv(), 256), 256, 0, (cudaStream_t)stream>>>(
      d, src, src_pitchT, dst, dst_pitchT, wsum, periodic, cw, 1.f, 1.f, 0.f, nullptr, nullptr);
  OTM_CHECK_LAUNCH("k_conv_forward");
  count_launches(1);
  return OTM_OK;
}

otm_status otm_filter_backward(const int reso[3], const float* g_dst, int g_dst_pitchT, const float* wsum,
                               float* g_src, int g_src_pitchT, int weight_type, float radius, int periodic,
                               void* stream) {
  OTM_TRY(check_reso(reso));
  if (!g_dst || !wsum || !g_src) return OTM_ERR_INVALID_ARGUMENT;
  const Dims d{reso[0], reso[1], reso[2]};
  if (g_dst_pitchT <= 0) g_dst_pitchT = d.nx;
  if (g_src_pitchT <= 0) g_src_pitchT = d.nx;
  if (g_dst_pitchT < d.nx || g_src_pitchT < d.nx) return OTM_ERR_INVALID_ARGUMENT;
  ConvWeights cw;
  OTM_TRY(make_weights(weight_type, radius, &cw));
  k_conv_backward<false><<<ceil_div(d.nv(), 256), 256, 0, (cudaStream_t)stream>>>(
      d, g_dst, g_dst_pitchT, nullptr, wsum, g_src, g_src_pitchT, periodic, cw);
  OTM_CHECK_LAUNCH("k_conv_backward");
  count_launches(1);
  return OTM_OK;
}

otm_status otm_density_forward(const int reso[3], const float* rho, int rho_pitchT, float* rho_f, float* k,
                               float* dk, float* wsum, int weight_type, float radius, int periodic, float p,
                               float k0, float kmin, void* stream) {
  OTM_TRY(check_reso(reso));
  if (!rho || !k || !dk || !wsum) return OTM_ERR_INVALID_ARGUMENT;
  const Dims d{reso[0], reso[1], reso[2]};
  if (rho_pitchT <= 0) rho_pitchT = d.nx;
  if (rho_pitchT < d.nx) return OTM_ERR_INVALID_ARGUMENT;
  ConvWeights cw;
  OTM_TRY(make_weights(weight_type, radius, &cw));
  k_conv_forward<true><<<ceil_div(d.nv(), 256), 256, 0, (cudaStream_t)stream>>>(
      d, rho, rho_pitchT, rho_f, d.nx, wsum, periodic, cw, p, k0, kmin, k, dk);
  OTM_CHECK_LAUNCH("k_conv_forward<simp>");
  count_launches(1);
  return OTM_OK;
}

otm_status otm_density_backward(const int reso[3], const float* g_k, const float* dk, const float* wsum,
                                float* g_rho, int g_rho_pitchT, int weight_type, float radius, int periodic,
                                void* stream) {
  OTM_TRY(check_reso(reso));
  if (!g_k || !dk || !wsum || !g_rho) return OTM_ERR_INVALID_ARGUMENT;
  const Dims d{reso[0], reso[1], reso[2]};
  if (g_rho_pitchT <= 0) g_rho_pitchT = d.nx;
  if (g_rho_pitchT < d.nx) return OTM_ERR_INVALID_ARGUMENT;
  ConvWeights cw;
  OTM_TRY(make_weights(weight_type, radius, &cw));
  k_conv_backward<true><<<ceil_div(d.nv(), 256), 256, 0, (cudaStream_t)stream>>>(
      d, g_k, d.nx, dk, wsum, g_rho, g_rho_pitchT, periodic, cw);
  OTM_CHECK_LAUNCH("k_conv_backward<chain>");
  count_launches(1);
  return OTM_OK;
}

}  // extern "C"
