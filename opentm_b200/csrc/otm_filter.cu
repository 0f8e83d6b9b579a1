// otm_filter.cu -- density filter (radial convolution with in-bounds renormalisation), the
// fused SIMP density chain and their adjoints (AutoDiff/TensorExpression.h:993-1185,
// AutoDiff/TensorExpression.cuh:281-385).
//
// The nonzero normalised weights travel as a kernel parameter (constant bank, broadcast to the
// warp), so no device allocation or global state is used.
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

// Shared-memory tiled convolution: a 256-thread block produces a 32 x 8 x 4 tile of outputs
// from the (32+2h) x (8+2h) x (4+2h) input tile it stages in shared memory (with periodic wrap
// or a validity mask for zero padding), so each input value is read from global memory about
// once instead of (2h+1)^3 times. The taps are summed in the reference's order (x fastest).
//   MODE 0: forward            out = sum w src / sum_valid w
//   MODE 1: forward + SIMP     also k = (k0 - kmin) out^p + kmin and dk = dk/dout
//   MODE 2: adjoint            out = sum_off w g(i - off) / ws(i - off)
//   MODE 3: adjoint chain      as 2 with g = g_k * dk
//   MODE 4: forward + SIMP + conductivity import: as 1, with k written as the solver's raw
//           conductivity and ks = 1e-9 + k^pp beside it (k_import's arithmetic), a negative,
//           NaN or Inf k flagged in *bad
constexpr int kTX = 32, kTY = 8, kTZ = 4;

template <int H>
constexpr int tile_elems() {
  return (kTX + 2 * H) * (kTY + 2 * H) * (kTZ + 2 * H);
}

// The nonzero taps of a filter in the reference's order (x fastest), each with its offset in
// the shared-memory tile: a radial kernel has many zero weights in its cube (27 of 125 taps are
// nonzero for radius 2), and skipping them leaves every sum unchanged.
struct TapList {
  int n;
  int doff[kMaxTaps];  // oz * SX * SY + oy * SX + ox for the forward direction (negated for the adjoint)
  float w[kMaxTaps];
};

template <int H>
static void make_taps(const ConvWeights& cw, TapList* tl) {
  constexpr int SX = kTX + 2 * H, SY = kTY + 2 * H, W1 = 2 * H + 1;
  tl->n = 0;
  for (int t = 0; t < cw.taps; t++) {
    if (cw.w[t] == 0.f) continue;
    const int ox = t % W1 - H, oy = t / W1 % W1 - H, oz = t / (W1 * W1) - H;
    tl->doff[tl->n] = oz * SX * SY + oy * SX + ox;
    tl->w[tl->n] = cw.w[t];
    tl->n++;
  }
}

template <int H, int MODE>
__global__ void __launch_bounds__(256) k_conv_tiled(Dims d, const float* __restrict__ src, int src_pitch,
                                                    const float* __restrict__ dk_in, const float* __restrict__ ws_in,
                                                    float* __restrict__ dst, int dst_pitch,
                                                    float* __restrict__ ws_out, int periodic, TapList tl,
                                                    float wsum_all, float p, float k0, float kmin,
                                                    float* __restrict__ kout, float* __restrict__ dkout,
                                                    float* __restrict__ ksout, float pp, int* bad) {
  constexpr int SX = kTX + 2 * H, SY = kTY + 2 * H, SZ = kTZ + 2 * H;
  constexpr bool kFwd = MODE < 2 || MODE == 4;
  extern __shared__ float sm[];
  float* val = sm;
  float* msk = sm + SX * SY * SZ;  // only used without periodicity
  const int x0 = blockIdx.x * kTX, y0 = blockIdx.y * kTY, z0 = blockIdx.z * kTZ;
  // stage the tile row by row: x from the thread's lane (two passes cover SX = 32 + 2H), the
  // (y, z) row from one small division, the wrapped x coordinates computed once
  int gxs[2];
  bool inx[2];
#pragma unroll
  for (int k = 0; k < 2; k++) {
    int gx = x0 + int(threadIdx.x) + k * kTX - H;
    inx[k] = gx >= 0 && gx < d.nx;
    if (!inx[k]) gx = ((gx % d.nx) + d.nx) % d.nx;
    gxs[k] = gx;
  }
  for (int rowi = threadIdx.y; rowi < SY * SZ; rowi += kTY) {
    const int ly = rowi % SY, lz = rowi / SY;
    int gy = y0 + ly - H, gz = z0 + lz - H;
    const bool inyz = gy >= 0 && gy < d.ny && gz >= 0 && gz < d.nz;
    if (gy < 0 || gy >= d.ny) gy = ((gy % d.ny) + d.ny) % d.ny;
    if (gz < 0 || gz >= d.nz) gz = ((gz % d.nz) + d.nz) % d.nz;
    const size_t row = size_t(gy) + size_t(d.ny) * gz;
#pragma unroll
    for (int k = 0; k < 2; k++) {
      const int lx = int(threadIdx.x) + k * kTX;
      if (lx >= SX) continue;
      const int gx = gxs[k];
      float v = 0.f, m = 0.f;
      if ((inx[k] && inyz) || periodic) {
        v = __ldg(src + row * src_pitch + gx);
        if (!kFwd) {
          const size_t q = row * d.nx + gx;
          if (MODE == 3) v *= __ldg(dk_in + q);
          v /= __ldg(ws_in + q);
        }
        m = 1.f;
      }
      val[rowi * SX + lx] = v;
      if (!periodic) msk[rowi * SX + lx] = m;
    }
  }
  __syncthreads();
  const int gx = x0 + threadIdx.x, gy = y0 + threadIdx.y;
  if (gx >= d.nx || gy >= d.ny) return;
  // the four z outputs of this thread together: each tap's weight and offset serve all four;
  // every output still sums its taps in the reference's order
  float sum[kTZ], wsv[kTZ];
#pragma unroll
  for (int tz = 0; tz < kTZ; tz++) sum[tz] = wsv[tz] = 0.f;
  const int base = H * SX * SY + (threadIdx.y + H) * SX + (threadIdx.x + H);
#pragma unroll 8
  for (int t = 0; t < tl.n; t++) {
    const float w = tl.w[t];
    const int li = base + (kFwd ? tl.doff[t] : -tl.doff[t]);
#pragma unroll
    for (int tz = 0; tz < kTZ; tz++) {
      sum[tz] += w * val[li + tz * SX * SY];
      if (kFwd && !periodic) wsv[tz] += w * msk[li + tz * SX * SY];
    }
  }
#pragma unroll
  for (int tz = 0; tz < kTZ; tz++) {
    const int gz = z0 + tz;
    if (gz >= d.nz) break;
    const float sumv = sum[tz];
    float ws = wsv[tz];
    const size_t row = size_t(gy) + size_t(d.ny) * gz;
    if (kFwd) {
      if (periodic) ws = wsum_all;
      const float out = sumv / ws;
      if (dst) dst[row * dst_pitch + gx] = out;
      if (ws_out) ws_out[row * d.nx + gx] = ws;
      if (MODE == 1 || MODE == 4) {
        const float pw = (p == 3.f) ? out * out * out : powf(out, p);
        const float k = (k0 - kmin) * pw + kmin;
        kout[row * d.nx + gx] = k;
        const float dpw = (p == 3.f) ? 3.f * out * out : p * powf(out, p - 1.f);
        dkout[row * d.nx + gx] = (k0 - kmin) * dpw;
        if (MODE == 4) {
          if (!(k >= 0.f) || !isfinite(k)) atomicOr(bad, 1);
          ksout[row * d.nx + gx] = kRhoPenalMin + (pp == 1.f ? k : powf(k, pp));
        }
      }
    } else {
      dst[row * dst_pitch + gx] = sumv;
    }
  }
}

template <int H, int MODE>
static otm_status launch_tiled(const Dims& d, const float* src, int src_pitch, const float* dk_in,
                               const float* ws_in, float* dst, int dst_pitch, float* ws_out, int periodic,
                               const ConvWeights& cw, float wsum_all, float p, float k0, float kmin, float* kout,
                               float* dkout, float* ksout, float pp, int* bad, cudaStream_t s) {
  const size_t smem = size_t(tile_elems<H>()) * sizeof(float) * (periodic ? 1 : 2);
  static bool attr = false;  // the attribute is per function and process-wide
  if (!attr) {
    cudaFuncSetAttribute(k_conv_tiled<H, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * tile_elems<H>() * 4);
    attr = true;
  }
  dim3 grid((d.nx + kTX - 1) / kTX, (d.ny + kTY - 1) / kTY, (d.nz + kTZ - 1) / kTZ);
  TapList tl;
  make_taps<H>(cw, &tl);
  k_conv_tiled<H, MODE><<<grid, dim3(kTX, kTY), smem, s>>>(d, src, src_pitch, dk_in, ws_in, dst, dst_pitch, ws_out,
                                                          periodic, tl, wsum_all, p, k0, kmin, kout, dkout, ksout,
                                                          pp, bad);
  OTM_CHECK_LAUNCH("k_conv_tiled");
  count_launches(1);
  return OTM_OK;
}

template <int MODE>
static otm_status conv_dispatch(const Dims& d, const float* src, int src_pitch, const float* dk_in,
                                const float* ws_in, float* dst, int dst_pitch, float* ws_out, int periodic,
                                const ConvWeights& cw, float p, float k0, float kmin, float* kout, float* dkout,
                                cudaStream_t s, float* ksout = nullptr, float pp = 1.f, int* bad = nullptr) {
  // sum of the normalised weights in the reference's tap order (the in-bounds weight of a
  // periodic filter)
  float wsum_all = 0.f;
  for (int t = 0; t < cw.taps; t++) wsum_all += cw.w[t];
  switch (cw.half) {
#define OTM_H(HH) \
  case HH:        \
    return launch_tiled<HH, MODE>(d, src, src_pitch, dk_in, ws_in, dst, dst_pitch, ws_out, periodic, cw, wsum_all, \
                                  p, k0, kmin, kout, dkout, ksout, pp, bad, s);
    OTM_H(0) OTM_H(1) OTM_H(2) OTM_H(3) OTM_H(4) OTM_H(5) OTM_H(6)
#undef OTM_H
  }
  set_error("unsupported filter half width");
  return OTM_ERR_UNSUPPORTED;
}

// The density chain's forward pass writing straight into a homogenization handle's conductivity
// buffers (otm_homo_update_density): rho_f, dk and wsum as otm_density_forward, k as kraw and
// ks = 1e-9 + k^pp, invalid values flagged in *bad.
otm_status density_forward_import(const Dims& d, const float* rho, int rho_pitchT, float* rho_f, float* dk,
                                  float* wsum, int weight_type, float radius, int periodic, float p, float k0,
                                  float kmin, float* kraw, float* ks, float pp, int* bad, cudaStream_t s) {
  if (!rho || !dk || !wsum) return OTM_ERR_INVALID_ARGUMENT;
  if (rho_pitchT <= 0) rho_pitchT = d.nx;
  if (rho_pitchT < d.nx) return OTM_ERR_INVALID_ARGUMENT;
  ConvWeights cw;
  OTM_TRY(make_weights(weight_type, radius, &cw));
  return conv_dispatch<4>(d, rho, rho_pitchT, nullptr, nullptr, rho_f, d.nx, wsum, periodic, cw, p, k0, kmin, kraw,
                          dk, s, ks, pp, bad);
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
  return conv_dispatch<0>(d, src, src_pitchT, nullptr, nullptr, dst, dst_pitchT, wsum, periodic, cw, 1.f, 1.f, 0.f,
                         nullptr, nullptr, (cudaStream_t)stream);
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
  return conv_dispatch<2>(d, g_dst, g_dst_pitchT, nullptr, wsum, g_src, g_src_pitchT, nullptr, periodic, cw, 1.f,
                         1.f, 0.f, nullptr, nullptr, (cudaStream_t)stream);
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
  return conv_dispatch<1>(d, rho, rho_pitchT, nullptr, nullptr, rho_f, d.nx, wsum, periodic, cw, p, k0, kmin, k, dk,
                         (cudaStream_t)stream);
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
  return conv_dispatch<3>(d, g_k, d.nx, dk, wsum, g_rho, g_rho_pitchT, nullptr, periodic, cw, 1.f, 1.f, 0.f, nullptr,
                         nullptr, (cudaStream_t)stream);
}

}  // extern "C"
