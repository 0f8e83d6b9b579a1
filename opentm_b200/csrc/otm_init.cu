// otm_init.cu -- initial density fields of the design loop and field symmetrisation.
//
// initDensity (Framework.cu:63-145): TPMS level sets (P, G, D, IWP) through the reference's
// tanh projection, the centred-sphere example, thresholded noise scaled to the volume ratio,
// and randTri (homogenization/Framework.cuh:237-310): a random trigonometric field whose
// sigmoid level set is bisected to the volume ratio. symetrize_tensor_kernel
// (AutoDiff/TensorExpression.cuh:70-280): orbit means under the reflection / rotation groups.
//
// All of it runs once per design run and is HBM-light; the kernels are one thread per cell (or
// per orbit), coalesced along x, with FP64 block reductions for the level-set bisection.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "opentm_b200_driver.h"
#include "otm_common.cuh"
#include "otm_driver_impl.h"

namespace otm {
namespace {

constexpr float kPiRef = 3.1415926f;  // the literal of Framework.cu:67 and Framework.cuh:110
constexpr int kInitBlock = 256;
constexpr int kMaxPeriod = 50;  // randTribase_sincos_kernel caps n_period at 50
constexpr int kInitMaxSmem = 200 * 1024;

// culib/lib.cuh:1372-1379
__device__ __forceinline__ float tanproj(float v, float beta, float tau) {
  const float tb = tanhf(beta * tau);
  return (tb + tanhf(beta * (v - tau))) / (tb + tanhf(beta * (1.f - tau)));
}

// culib/lib.cuh:1381-1383
__device__ __forceinline__ float sigmoid_ref(float v, float k, float center) {
  return 1.f / (1.f + expf(-k * (v - center)));
}

__device__ __forceinline__ size_t at(const Dims& d, int pitchT, int x, int y, int z) {
  return (size_t(z) * d.ny + y) * size_t(pitchT) + x;
}

// value i of stream seed in [0, 1), 53 bits (opentm_b200/workloads.py `uniform`)
__host__ __device__ __forceinline__ double uniform01(uint64_t seed, uint64_t i) {
  uint64_t z = (seed << 32) + i;
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return double(z >> 11) * (1.0 / 9007199254740992.0);
}

// ---------------------------------------------------------------------------------------
// Closed-form initial fields (Framework.cu:86-139)
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kInitBlock) k_init_closed(Dims d, int pitchT, int way, float* out) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= d.nv()) return;
  const Coord3 c = split3(e, d.nx, d.ny);
  const float p0 = float(c.x) / d.nx, p1 = float(c.y) / d.ny, p2 = float(c.z) / d.nz;
  float v = 0.f;
  if (way == OTM_INIT_P) {
    const float val = cosf(2 * kPiRef * p0) + cosf(2 * kPiRef * p1) + cosf(2 * kPiRef * p2);
    v = fmaxf(fminf(tanproj(-val, 20.f, 0.5f), 1.f), 0.001f);
  } else if (way == OTM_INIT_G) {
    const float p[3] = {p0, p1, p2};
    float s[3], co[3];
    for (int i = 0; i < 3; i++) {
      s[i] = sinf(2 * kPiRef * p[i]);
      co[i] = cosf(2 * kPiRef * p[i]);
    }
    const float val = s[0] * co[1] + s[2] * co[0] + s[1] * co[2];
    v = fmaxf(fminf(tanproj(val, 20.f, 0.5f), 1.f), 0.001f);
  } else if (way == OTM_INIT_D) {
    const float x = p0, y = p1, z = p2;
    const float val = cosf(2 * kPiRef * x) * cosf(2 * kPiRef * y) * cosf(2 * kPiRef * z) -
                      sinf(2 * kPiRef * x) * sinf(2 * kPiRef * y) * sinf(2 * kPiRef * z);
    v = fmaxf(fminf(tanproj(val, 20.f, 0.5f), 1.f), 0.001f);
  } else if (way == OTM_INIT_IWP) {
    const float x = p0, y = p1, z = p2;
    const float val = 2 * (cosf(2 * kPiRef * x) * cosf(2 * kPiRef * y) + cosf(2 * kPiRef * y) * cosf(2 * kPiRef * z) +
                           cosf(2 * kPiRef * z) * cosf(2 * kPiRef * x)) -
                      (cosf(2 * 2 * kPiRef * x) + cosf(2 * 2 * kPiRef * y) + cosf(2 * 2 * kPiRef * z));
    v = fmaxf(fminf(tanproj(val, 20.f, 0.5f), 1.f), 0.001f);
  } else {  // OTM_INIT_EXAMPLE: a void sphere of radius min(reso)/6 at the centre, 0.3 elsewhere
    const double dx = c.x - double(d.nx) / 2 + 0.5, dy = c.y - double(d.ny) / 2 + 0.5,
                 dz = c.z - double(d.nz) / 2 + 0.5;
    const double r = double(min(min(d.nx, d.ny), d.nz)) / 6.0;
    v = sqrt(dx * dx + dy * dy + dz * dz) < r ? 0.f : 0.3f;
  }
  out[at(d, pitchT, c.x, c.y, c.z)] = v;
}

// Tensor::rand(0, 1) with the library's stream: cell e takes value e of stream `seed`.
__global__ void __launch_bounds__(kInitBlock) k_noise(Dims d, int pitchT, uint64_t seed, float* out) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= d.nv()) return;
  const Coord3 c = split3(e, d.nx, d.ny);
  out[at(d, pitchT, c.x, c.y, c.z)] = float(uniform01(seed, e));
}

// Tensor::proj(20, 0.5) (projectTensor_kernel, AutoDiff/TensorExpression.cu:105-115)
__global__ void __launch_bounds__(kInitBlock) k_proj(Dims d, int pitchT, float beta, float tau, float* f) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= d.nv()) return;
  const Coord3 c = split3(e, d.nx, d.ny);
  const size_t i = at(d, pitchT, c.x, c.y, c.z);
  float rho = tanproj(f[i], beta, tau);
  if (rho < 0.5f) rho = 1e-9f;
  if (rho > 0.5f) rho = 1.f;
  f[i] = rho;
}

// newval = val * s clamped to [0.001, 1] (Framework.cu:79-84)
__global__ void __launch_bounds__(kInitBlock) k_scale_clamp(Dims d, int pitchT, const double* mean, float vol,
                                                            float* f) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= d.nv()) return;
  const float s = vol / float(*mean);
  const Coord3 c = split3(e, d.nx, d.ny);
  const size_t i = at(d, pitchT, c.x, c.y, c.z);
  float v = f[i] * s;
  if (v < 0.001f) v = 0.001f;
  if (v >= 1.f) v = 1.f;
  f[i] = v;
}

// Tensor::clamp(low, upp) (AutoDiff/TensorExpression.h:492-502)
__global__ void __launch_bounds__(kInitBlock) k_clamp(Dims d, int pitchT, float lo, float hi, float* f) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= d.nv()) return;
  const Coord3 c = split3(e, d.nx, d.ny);
  const size_t i = at(d, pitchT, c.x, c.y, c.z);
  const float v = f[i];
  f[i] = v < lo ? lo : (v > hi ? hi : (v >= lo && v <= hi ? v : lo));
}

// ---------------------------------------------------------------------------------------
// Random trigonometric basis (randTribase_sincos_kernel, Framework.cuh:106-215)
// ---------------------------------------------------------------------------------------
// g holds the 6n one-dimensional functions in the second-order ordering: j < 3n is
// cos(2 pi (j % n + 1) p[j / n]), j >= 3n is sin(2 pi (j % n + 1) p[j / n - 3]). First-order
// term i < 3n uses cos of axis i % 3 and frequency i / 3; i in [3n, 6n) the sin of
// (i - 3n) % 3, (i - 3n) / 3. Second-order term 6n + j * 6n + k is g_j g_k.
// The products are FP32 like the reference's; they are accumulated in FP64, so the field does not
// depend on the summation order (the reference sums warp-strided partials in FP32).
__global__ void __launch_bounds__(kInitBlock) k_randtri(Dims d, int pitchT, int n, const float* __restrict__ coeff,
                                                        int staged, int centered, const float* __restrict__ rot,
                                                        float* out) {
  extern __shared__ float sc[];  // the coefficients, staged once per block when they fit
  const int nb1 = 6 * n, nb = nb1 + 36 * n * n;
  if (staged) {
    for (int i = threadIdx.x; i < nb; i += blockDim.x) sc[i] = coeff[i];
    __syncthreads();
  }
  const float* cs = staged ? sc : coeff;
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= d.nv()) return;
  const Coord3 c = split3(e, d.nx, d.ny);
  float p[3] = {c.x / (float(d.nx) - 1.f), c.y / (float(d.ny) - 1.f), c.z / (float(d.nz) - 1.f)};
  if (centered) {
    const float q0 = p[0] - 0.5f, q1 = p[1] - 0.5f, q2 = p[2] - 0.5f;
    p[0] = rot[0] * q0 + rot[1] * q1 + rot[2] * q2;
    p[1] = rot[3] * q0 + rot[4] * q1 + rot[5] * q2;
    p[2] = rot[6] * q0 + rot[7] * q1 + rot[8] * q2;
  }
  constexpr float pi2 = kPiRef * 2;
  float g[6 * kMaxPeriod];
  for (int a = 0; a < 3; a++)
    for (int f = 0; f < n; f++) {
      g[a * n + f] = cosf(pi2 * (f + 1) * p[a]);
      g[3 * n + a * n + f] = sinf(pi2 * (f + 1) * p[a]);
    }
  double s = 0.0;
  for (int i = 0; i < nb1; i++) {
    const int ii = i < 3 * n ? i : i - 3 * n;
    s += double(cs[i] * g[(i < 3 * n ? 0 : 3 * n) + (ii % 3) * n + ii / 3]);
  }
  for (int j = 0; j < nb1; j++) {
    const float* cj = cs + nb1 + size_t(j) * nb1;
    const float gj = g[j];
    for (int k = 0; k < nb1; k++) s += double(cj[k] * gj * g[k]);
  }
  out[at(d, pitchT, c.x, c.y, c.z)] = float(s);
}

// sigmoid level set mapped to [m, M] (Framework.cuh:286-294)
__device__ __forceinline__ float level_map(float val, float t, float M, float m) {
  return sigmoid_ref(val, 15.f, t) * (M - m) + m;
}

// Partial sums of the field (mode 0) or of its level-set map at t (mode 1): one FP64 value per
// block, reduced in a fixed order by k_final_sum.
__global__ void __launch_bounds__(kInitBlock) k_partial_sum(Dims d, int pitchT, const float* __restrict__ f,
                                                            int mode, float t, float M, float m, double* part) {
  __shared__ double sm[32];
  double v[1] = {0.0};
  const size_t nv = d.nv();
  for (size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x; e < nv; e += size_t(gridDim.x) * blockDim.x) {
    const Coord3 c = split3(e, d.nx, d.ny);
    const float x = f[at(d, pitchT, c.x, c.y, c.z)];
    v[0] += mode ? double(level_map(x, t, M, m)) : double(x);
  }
  block_reduce_f64<1>(v, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = v[0];
}

__global__ void __launch_bounds__(1024) k_final_sum(const double* __restrict__ part, int n, double scale,
                                                    double* out) {
  __shared__ double sm[32];
  double v[1] = {0.0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) v[0] += part[i];
  block_reduce_f64<1>(v, sm);
  if (threadIdx.x == 0) *out = v[0] * scale;
}

__global__ void __launch_bounds__(kInitBlock) k_level_map(Dims d, int pitchT, float t, float M, float m, float* f) {
  const size_t e = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= d.nv()) return;
  const Coord3 c = split3(e, d.nx, d.ny);
  const size_t i = at(d, pitchT, c.x, c.y, c.z);
  f[i] = level_map(f[i], t, M, m);
}

// ---------------------------------------------------------------------------------------
// Symmetrisation (symetrize_tensor_kernel, AutoDiff/TensorExpression.cuh:70-280)
// ---------------------------------------------------------------------------------------
// REFLECT3: representatives [0, n/2)^3; orbit = the 8 corner mirrors (flip bits i%2, i/2%2, i/4).
__global__ void __launch_bounds__(kInitBlock) k_sym_reflect3(Dims d, int pitchT, int average, float* f) {
  const int hx = d.nx / 2, hy = d.ny / 2, hz = d.nz / 2;
  const size_t tid = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (tid >= size_t(hx) * hy * hz) return;
  const int r[3] = {int(tid % hx), int(tid / hx % hy), int(tid / (size_t(hx) * hy))};
  const int n[3] = {d.nx, d.ny, d.nz};
  size_t idx[8];
  for (int i = 0; i < 8; i++) {
    const int fl[3] = {i % 2, i / 2 % 2, i / 4};
    int o[3];
    for (int j = 0; j < 3; j++) o[j] = fl[j] ? n[j] - 1 - r[j] : r[j];
    idx[i] = at(d, pitchT, o[0], o[1], o[2]);
  }
  float v = f[idx[0]];
  if (average) {
    for (int i = 1; i < 8; i++) v += f[idx[i]];
    v /= 8;
  }
  for (int i = 0; i < 8; i++) f[idx[i]] = v;
}

// REFLECT6 (cube): representatives x <= y <= z < n/2; orbit = 8 mirrors x 6 permutations, in
// the reference's order [a,b,c], [a,c,b], [c,a,b], [c,b,a], [b,a,c], [b,c,a].
__global__ void __launch_bounds__(kInitBlock) k_sym_reflect6(Dims d, int pitchT, float* f) {
  const int h = d.nx / 2;
  const size_t tid = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (tid >= size_t(h) * (h + 1) * (h + 2) / 6) return;
  // z = largest k with k (k+1) (k+2) / 6 <= tid; then y = largest j with j (j+1) / 2 <= rest
  long long z = llround(cbrt(6.0 * double(tid)));
  while (z > 0 && z * (z + 1) * (z + 2) / 6 > (long long)tid) z--;
  while ((z + 1) * (z + 2) * (z + 3) / 6 <= (long long)tid) z++;
  long long rest = (long long)tid - z * (z + 1) * (z + 2) / 6;
  long long y = llround(sqrt(2.0 * double(rest)));
  while (y > 0 && y * (y + 1) / 2 > rest) y--;
  while ((y + 1) * (y + 2) / 2 <= rest) y++;
  const int rx = int(rest - y * (y + 1) / 2), ry = int(y), rz = int(z);
  if (rz >= h || ry > rz || rx > ry) return;  // cannot happen for tid in range
  const int n = d.nx;
  float sum = 0.f;
  for (int pass = 0; pass < 2; pass++) {
    for (int i = 0; i < 8; i++) {
      const int a = (i % 2) ? n - 1 - rx : rx, b = (i / 2 % 2) ? n - 1 - ry : ry, c = (i / 4) ? n - 1 - rz : rz;
      const size_t pts[6] = {at(d, pitchT, a, b, c), at(d, pitchT, a, c, b), at(d, pitchT, c, a, b),
                             at(d, pitchT, c, b, a), at(d, pitchT, b, a, c), at(d, pitchT, b, c, a)};
      for (int k = 0; k < 6; k++) {
        if (pass == 0)
          sum += f[pts[k]];
        else
          f[pts[k]] = sum;
      }
    }
    if (pass == 0) sum /= 48;  // this branch of the reference averages whatever `average` says
  }
}

// ROTATE3 (even cube): the 24 rotations about the centre. Offsets o >= 0 from the centre plane
// h = n/2: coordinate h + o (positive side) or h - 1 - o (mirrored). Representatives
// max(x, y) <= z < h. Odd permutations take one or three mirrored axes, even ones zero or two.
// Representatives that are cyclic rotations of one another share an orbit; only the first of
// them in enumeration order writes it.
__global__ void __launch_bounds__(kInitBlock) k_sym_rotate3(Dims d, int pitchT, float* f) {
  const int h = d.nx / 2;
  const size_t tid = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (tid >= size_t(h) * (h + 1) * (2 * h + 1) / 6) return;
  // z = largest k with k (k+1) (2k+1) / 6 <= tid
  long long z = llround(cbrt(3.0 * double(tid)));
  while (z > 0 && z * (z + 1) * (2 * z + 1) / 6 > (long long)tid) z--;
  while ((z + 1) * (z + 2) * (2 * z + 3) / 6 <= (long long)tid) z++;
  const long long rest = (long long)tid - z * (z + 1) * (2 * z + 1) / 6;
  const int rz = int(z), ry = int(rest / (z + 1)), rx = int(rest % (z + 1));
  if (rz >= h || rx > rz || ry > rz) return;  // cannot happen for tid in range
  // canonical representative of the orbit: the cyclic rotations (z, x, y) and (y, z, x) are
  // representatives too when they satisfy max(first two) <= third; the one with the smallest
  // in-layer key y (z + 1) + x writes
  const long long key = (long long)ry * (rz + 1) + rx;
  if (rx == rz && (long long)rz * (rz + 1) + ry < key) return;  // (y, z, x) with x == z
  if (ry == rz && (long long)rx * (rz + 1) + rz < key) return;  // (z, x, y) with y == z
  const int rep[3] = {rx, ry, rz};
  const int perm[6][3] = {{0, 2, 1}, {2, 1, 0}, {1, 0, 2}, {2, 0, 1}, {1, 2, 0}, {0, 1, 2}};
  float sum = 0.f;
  for (int pass = 0; pass < 2; pass++) {
    for (int i = 0; i < 6; i++) {
      const int o0 = rep[perm[i][0]], o1 = rep[perm[i][1]], o2 = rep[perm[i][2]];
      const int P0 = h + o0, P1 = h + o1, P2 = h + o2, M0 = h - 1 - o0, M1 = h - 1 - o1, M2 = h - 1 - o2;
      size_t pts[4];
      if (i < 3) {
        pts[0] = at(d, pitchT, M0, P1, P2);
        pts[1] = at(d, pitchT, P0, M1, P2);
        pts[2] = at(d, pitchT, P0, P1, M2);
        pts[3] = at(d, pitchT, M0, M1, M2);
      } else {
        pts[0] = at(d, pitchT, P0, P1, P2);
        pts[1] = at(d, pitchT, M0, M1, P2);
        pts[2] = at(d, pitchT, P0, M1, M2);
        pts[3] = at(d, pitchT, M0, P1, M2);
      }
      for (int k = 0; k < 4; k++) {
        if (pass == 0)
          sum += f[pts[k]];
        else
          f[pts[k]] = sum;
      }
    }
    if (pass == 0) sum /= 24;  // likewise always averaged
  }
}

// ROTATE2: representatives x < nx/2; orbit = {p, mirror of p through the centre}.
__global__ void __launch_bounds__(kInitBlock) k_sym_rotate2(Dims d, int pitchT, int average, float* f) {
  const int hx = d.nx / 2;
  const size_t tid = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (tid >= size_t(hx) * d.ny * d.nz) return;
  const int x = int(tid % hx), y = int(tid / hx % d.ny), z = int(tid / (size_t(hx) * d.ny));
  const size_t a = at(d, pitchT, x, y, z), b = at(d, pitchT, d.nx - 1 - x, d.ny - 1 - y, d.nz - 1 - z);
  float v = f[a];
  if (average) {
    v += f[b];
    v /= 2;
  }
  f[a] = v;
  f[b] = v;
}

constexpr int kSumBlocks = 296;  // two blocks per SM; fixed, so sums are reproducible

otm_status check_field(const int reso[3], int* pitchT) {
  if (!reso) return OTM_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < 3; i++)
    if (reso[i] < 1 || reso[i] > 1024) {
      set_error("field sizes must be 1..1024 per axis");
      return OTM_ERR_INVALID_ARGUMENT;
    }
  if (*pitchT <= 0) *pitchT = reso[0];
  if (*pitchT < reso[0]) {
    set_error("pitchT smaller than the x resolution");
    return OTM_ERR_INVALID_ARGUMENT;
  }
  return OTM_OK;
}

// Mean of the field (mode 0) or of its level-set map (mode 1) into *out_dev; launches only.
void launch_mean(Dims d, int pitchT, const float* f, int mode, float t, float M, float m, double* part,
                 double* out_dev, cudaStream_t s) {
  k_partial_sum<<<kSumBlocks, kInitBlock, 0, s>>>(d, pitchT, f, mode, t, M, m, part);
  k_final_sum<<<1, 1024, 0, s>>>(part, kSumBlocks, 1.0 / double(d.nv()), out_dev);
  count_launches(2);
}

// glm::toMat3(normalize(quat(w, x, y, z))) as a row-major matrix acting on column vectors
void quat_rotation(const float q[4], float R[9]) {
  double w = q[0], x = q[1], y = q[2], z = q[3];
  const double nrm = std::sqrt(w * w + x * x + y * y + z * z);
  if (nrm > 0) {
    w /= nrm;
    x /= nrm;
    y /= nrm;
    z /= nrm;
  } else {
    w = 1;
    x = y = z = 0;
  }
  R[0] = float(1 - 2 * (y * y + z * z));
  R[1] = float(2 * (x * y - w * z));
  R[2] = float(2 * (x * z + w * y));
  R[3] = float(2 * (x * y + w * z));
  R[4] = float(1 - 2 * (x * x + z * z));
  R[5] = float(2 * (y * z - w * x));
  R[6] = float(2 * (x * z - w * y));
  R[7] = float(2 * (y * z + w * x));
  R[8] = float(1 - 2 * (x * x + y * y));
}

}  // namespace

otm_status field_means(const int reso[3], const float* a, const float* b, int pitchT, cudaStream_t s,
                       double out[2]) {
  const Dims d{reso[0], reso[1], reso[2]};
  double* dev = nullptr;
  double* host = nullptr;
  cudaError_t e = scratch_malloc((void**)&dev, (2 * kSumBlocks + 2) * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&host, 2 * sizeof(double));
  if (e == cudaSuccess) {
    launch_mean(d, pitchT, a, 0, 0.f, 0.f, 0.f, dev, dev + 2 * kSumBlocks, s);
    launch_mean(d, pitchT, b, 0, 0.f, 0.f, 0.f, dev + kSumBlocks, dev + 2 * kSumBlocks + 1, s);
    e = cudaMemcpyAsync(host, dev + 2 * kSumBlocks, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
  }
  if (dev) cudaFreeAsync(dev, s);
  const cudaError_t e2 = cudaStreamSynchronize(s);
  if (e == cudaSuccess && e2 == cudaSuccess) {
    out[0] = host[0];
    out[1] = host[1];
  }
  if (host) cudaFreeHost(host);
  if (e != cudaSuccess) return cuda_fail(e, "field mean");
  if (e2 != cudaSuccess) return cuda_fail(e2, "field mean");
  return OTM_OK;
}

otm_status symmetrize_field(const int reso[3], float* f, int pitchT, int sym, int average, cudaStream_t s) {
  if (sym == OTM_SYM_NONE) return OTM_OK;
  const Dims d{reso[0], reso[1], reso[2]};
  size_t nrep = 0;
  if (sym == OTM_SYM_REFLECT3) {
    nrep = size_t(d.nx / 2) * (d.ny / 2) * (d.nz / 2);
  } else if (sym == OTM_SYM_REFLECT6 || sym == OTM_SYM_ROTATE3) {
    if (d.nx != d.ny || d.nx != d.nz || (sym == OTM_SYM_ROTATE3 && d.nx % 2)) {
      set_error(sym == OTM_SYM_REFLECT6 ? "reflect6 symmetry needs a cubic cell" : "rotate3 symmetry needs an even cube");
      return OTM_ERR_UNSUPPORTED;
    }
    const size_t h = d.nx / 2;
    nrep = sym == OTM_SYM_REFLECT6 ? h * (h + 1) * (h + 2) / 6 : h * (h + 1) * (2 * h + 1) / 6;
  } else if (sym == OTM_SYM_ROTATE2) {
    nrep = size_t(d.nx / 2) * d.ny * d.nz;
  } else {
    set_error("unknown symmetry");
    return OTM_ERR_INVALID_ARGUMENT;
  }
  if (nrep == 0) return OTM_OK;
  const int grid = ceil_div(nrep, kInitBlock);
  if (sym == OTM_SYM_REFLECT3) k_sym_reflect3<<<grid, kInitBlock, 0, s>>>(d, pitchT, average, f);
  if (sym == OTM_SYM_REFLECT6) k_sym_reflect6<<<grid, kInitBlock, 0, s>>>(d, pitchT, f);
  if (sym == OTM_SYM_ROTATE3) k_sym_rotate3<<<grid, kInitBlock, 0, s>>>(d, pitchT, f);
  if (sym == OTM_SYM_ROTATE2) k_sym_rotate2<<<grid, kInitBlock, 0, s>>>(d, pitchT, average, f);
  OTM_CHECK_LAUNCH("symmetrize");
  count_launches(1);
  return OTM_OK;
}

}  // namespace otm

using namespace otm;

extern "C" {

size_t otm_randtri_coeff_count(int n_period, int centered) {
  if (n_period < 1) return 0;
  if (n_period > kMaxPeriod) n_period = kMaxPeriod;
  return size_t(6) * n_period + size_t(36) * n_period * n_period + (centered ? 4 : 0);
}

otm_status otm_randtri_coefficients(uint64_t seed, int n_period, int centered, float* coeffs_host) {
  if (!coeffs_host || n_period < 1) return OTM_ERR_INVALID_ARGUMENT;
  const size_t n = otm_randtri_coeff_count(n_period, centered);
  for (size_t i = 0; i < n; i++) coeffs_host[i] = float(-1.0 + 2.0 * uniform01(seed, i));
  return OTM_OK;
}

otm_status otm_symmetrize(const int reso[3], float* field, int pitchT, int sym, int average, void* stream) {
  if (!field) return OTM_ERR_INVALID_ARGUMENT;
  OTM_TRY(check_field(reso, &pitchT));
  return symmetrize_field(reso, field, pitchT, sym, average, (cudaStream_t)stream);
}

otm_status otm_randtri_field(const int reso[3], float* field, int pitchT, int n_period, const float* coeffs_host,
                             int centered, void* stream) {
  if (!field || !coeffs_host || n_period < 1) return OTM_ERR_INVALID_ARGUMENT;
  OTM_TRY(check_field(reso, &pitchT));
  if (n_period > kMaxPeriod) n_period = kMaxPeriod;
  cudaStream_t s = (cudaStream_t)stream;
  const Dims d{reso[0], reso[1], reso[2]};
  const size_t nb = otm_randtri_coeff_count(n_period, 0);
  float R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (centered) quat_rotation(coeffs_host + nb, R);
  // coefficients then the rotation, in one upload from pinned memory
  float* h = nullptr;
  OTM_CUDA(cudaMallocHost((void**)&h, (nb + 9) * sizeof(float)));
  std::memcpy(h, coeffs_host, nb * sizeof(float));
  std::memcpy(h + nb, R, 9 * sizeof(float));
  float* dbuf = nullptr;
  cudaError_t e = scratch_malloc((void**)&dbuf, (nb + 9) * sizeof(float), s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dbuf, h, (nb + 9) * sizeof(float), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    // coefficients in shared memory when they fit (n_period <= 37), else read through L1
    const size_t smem = nb * sizeof(float);
    const int staged = smem <= size_t(kInitMaxSmem);
    const int grid = ceil_div(d.nv(), kInitBlock);
    if (staged && smem > 48 * 1024)
      e = cudaFuncSetAttribute(k_randtri, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kInitMaxSmem));
    if (e == cudaSuccess) {
      k_randtri<<<grid, kInitBlock, staged ? smem : 0, s>>>(d, pitchT, n_period, dbuf, staged, centered, dbuf + nb,
                                                            field);
      e = cudaGetLastError();
      count_launches(1);
    }
  }
  if (dbuf) cudaFreeAsync(dbuf, s);
  const cudaError_t e2 = cudaStreamSynchronize(s);  // the pinned upload buffer is free after this
  cudaFreeHost(h);
  if (e != cudaSuccess) return cuda_fail(e, "otm_randtri_field");
  if (e2 != cudaSuccess) return cuda_fail(e2, "otm_randtri_field");
  return OTM_OK;
}

otm_status otm_init_density(const otm_driver_config* cfg, float* rho, int pitchT, float* coeffs_out, void* stream) {
  if (!cfg || !rho) return OTM_ERR_INVALID_ARGUMENT;
  const int reso[3] = {cfg->reso, cfg->reso, cfg->reso};
  OTM_TRY(check_field(reso, &pitchT));
  cudaStream_t s = (cudaStream_t)stream;
  const Dims d{cfg->reso, cfg->reso, cfg->reso};
  const size_t nv = d.nv();
  const int grid = ceil_div(nv, kInitBlock);
  const int w = cfg->winit;
  double* dsum = nullptr;  // kSumBlocks partials, then the result
  double* hsum = nullptr;
  auto cleanup = [&]() {
    if (dsum) cudaFreeAsync(dsum, s);
    cudaStreamSynchronize(s);
    if (hsum) cudaFreeHost(hsum);
  };
  auto mean_now = [&](int mode, float t, float M, float m, double* out) -> otm_status {
    launch_mean(d, pitchT, rho, mode, t, M, m, dsum, dsum + kSumBlocks, s);
    OTM_CUDA(cudaMemcpyAsync(hsum, dsum + kSumBlocks, sizeof(double), cudaMemcpyDeviceToHost, s));
    OTM_CUDA(cudaStreamSynchronize(s));
    *out = *hsum;
    return OTM_OK;
  };
  otm_status st = OTM_OK;
  if (cudaMallocHost((void**)&hsum, sizeof(double)) != cudaSuccess ||
      scratch_malloc((void**)&dsum, (kSumBlocks + 1) * sizeof(double), s) != cudaSuccess) {
    cleanup();
    set_error("otm_init_density: out of memory");
    return OTM_ERR_OUT_OF_MEMORY;
  }
  if (w == OTM_INIT_P || w == OTM_INIT_G || w == OTM_INIT_D || w == OTM_INIT_IWP || w == OTM_INIT_EXAMPLE) {
    k_init_closed<<<grid, kInitBlock, 0, s>>>(d, pitchT, w, rho);
    count_launches(1);
  } else if (w == OTM_INIT_NOISE) {
    k_noise<<<grid, kInitBlock, 0, s>>>(d, pitchT, cfg->seed, rho);
    count_launches(1);
    st = symmetrize_field(reso, rho, pitchT, cfg->sym, 1, s);
    if (st == OTM_OK) {
      k_proj<<<grid, kInitBlock, 0, s>>>(d, pitchT, 20.f, 0.5f, rho);
      count_launches(1);
      launch_mean(d, pitchT, rho, 0, 0.f, 0.f, 0.f, dsum, dsum + kSumBlocks, s);
      k_scale_clamp<<<grid, kInitBlock, 0, s>>>(d, pitchT, dsum + kSumBlocks, float(cfg->vol_ratio), rho);
      count_launches(1);
    }
  } else if (w == OTM_INIT_RANDOM || w == OTM_INIT_RANDCENTER || w == OTM_INIT_REP_RANDCENTER) {
    // randTri (Framework.cuh:237-310)
    const int n = std::min(std::max(cfg->init_period, 1), kMaxPeriod);
    const int centered = w != OTM_INIT_RANDOM;
    const size_t nb = otm_randtri_coeff_count(n, centered);
    std::vector<float> co(nb);
    if (w == OTM_INIT_REP_RANDCENTER) {
      size_t len = 0;
      float* vec = co.data();
      st = cfg->input_path ? otm_read_vectors(cfg->input_path, 1, &len, &vec, nb) : OTM_ERR_INVALID_ARGUMENT;
      if (st == OTM_OK && len != nb) {
        set_error("coefficient file does not match the basis size");
        st = OTM_ERR_INVALID_ARGUMENT;
      }
    } else {
      st = otm_randtri_coefficients(cfg->seed, n, centered, co.data());
    }
    if (st == OTM_OK && coeffs_out) std::memcpy(coeffs_out, co.data(), nb * sizeof(float));
    if (st == OTM_OK) st = otm_randtri_field(reso, rho, pitchT, n, co.data(), centered, s);
    if (st == OTM_OK) st = symmetrize_field(reso, rho, pitchT, cfg->sym, 1, s);
    // level set: bisection on t until the mapped mean is within 1e-3 (relative) of the goal
    const float vol = float(cfg->vol_ratio);
    const float M = std::min(vol * 1.5f, 1.f), m = 0.001f;
    float t_u = float(n * n * 37), t_l = -t_u, t = (t_u + t_l) / 2;
    for (int it = 0; st == OTM_OK && it < 60; it++) {
      t = (t_u + t_l) / 2;
      double mean = 0;
      st = mean_now(1, t, M, m, &mean);
      if (st != OTM_OK) break;
      const float sv = float(mean);
      if (std::fabs(sv - vol) / vol < 1e-3f) break;
      if (sv > vol) t_l = t;
      if (sv < vol) t_u = t;
    }
    if (st == OTM_OK) {
      k_level_map<<<grid, kInitBlock, 0, s>>>(d, pitchT, t, M, m, rho);
      count_launches(1);
    }
  } else if (w == OTM_INIT_MANUAL) {
    int r3[3] = {0, 0, 0};
    std::vector<float> host;
    st = cfg->input_path ? otm_read_density_binary(cfg->input_path, r3, nullptr, 0) : OTM_ERR_INVALID_ARGUMENT;
    if (st == OTM_OK && (r3[0] != d.nx || r3[1] != d.ny || r3[2] != d.nz)) {
      set_error("density file resolution differs from the configured one");
      st = OTM_ERR_INVALID_ARGUMENT;
    }
    if (st == OTM_OK) {
      host.resize(nv);
      st = otm_read_density_binary(cfg->input_path, r3, host.data(), nv);
    }
    if (st == OTM_OK) {
      const cudaError_t e = cudaMemcpy2DAsync(rho, size_t(pitchT) * sizeof(float), host.data(),
                                              size_t(d.nx) * sizeof(float), size_t(d.nx) * sizeof(float),
                                              size_t(d.ny) * d.nz, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) st = cuda_fail(e, "density upload");
      else if (cudaStreamSynchronize(s) != cudaSuccess) st = cuda_fail(cudaGetLastError(), "density upload");
    }
  } else if (w == OTM_INIT_INTERP) {
    set_error("interp initialisation resamples an OpenVDB grid; OpenVDB is not supported");
    st = OTM_ERR_UNSUPPORTED;
  } else {
    set_error("unknown initialisation");
    st = OTM_ERR_INVALID_ARGUMENT;
  }
  // symmetrize, then clamp to [0.1, 1] (Framework.cu:140-144)
  if (st == OTM_OK) st = symmetrize_field(reso, rho, pitchT, cfg->sym, 1, s);
  if (st == OTM_OK) {
    k_clamp<<<grid, kInitBlock, 0, s>>>(d, pitchT, 0.1f, 1.f, rho);
    count_launches(1);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) st = cuda_fail(e, "otm_init_density");
  }
  cleanup();
  if (st == OTM_OK) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "otm_init_density");
  }
  return st;
}

}  // extern "C"
