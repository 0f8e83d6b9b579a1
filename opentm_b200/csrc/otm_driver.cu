// otm_driver.cu -- the tensor-matching design loop (runCustom, Framework.cu:147-244) with its
// convergence test and volume governor (homogenization/Framework.cuh:312-411), and the driver's
// file formats (homogenization/utils.h:47-91, grid.cpp:336-344, homoExpression.h:130-146).
//
// The loop is host orchestration over the library's device entry points on one stream: every
// field stays resident in HBM for the whole run; per iteration the host reads back only K^H (nine
// doubles, from the solve) and two field means (for the volume governor).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "opentm_b200_driver.h"
#include "opentm_b200_mma.h"
#include "otm_common.cuh"
#include "otm_driver_impl.h"

namespace otm {
namespace {

// ConvergeChecker::cirId (Framework.cuh:320-323)
int cir_id(int id) {
  while (id < 0) id += 10;
  return id % 10;
}

// VolumeGovernor::shrink / expand (Framework.cuh:357-365)
void gov_shrink(otm_volume_governor* g) {
  g->decrease = g->volume_bound - g->low_bound;
  g->volume_bound = g->volume_bound - g->decrease_factor * g->decrease;
  if (g->decrease_factor > 0.05) g->decrease_factor *= 0.8;
}
void gov_expand(otm_volume_governor* g) { g->volume_bound += 0.3 * g->decrease * g->decrease_factor; }

// The objective of runCustom (Framework.cu:168-170), in FP32 like the reference's expression:
// (K00 - t0)^2 + (K11 - t1)^2 + (K22 - t2)^2 + (K01 - t3)^2 + (K21 - t4)^2 + (K02 - t5)^2 - 1e-4,
// and its gradient with respect to K (the entries of gradH_ that the expression touches).
const int kObjEntry[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {2, 1}, {0, 2}};
float objective(const float K[9], const double t[6], float dK[9]) {
  float v = 0.f;
  for (int i = 0; i < 9; i++) dK[i] = 0.f;
  for (int e = 0; e < 6; e++) {
    const int ij = kObjEntry[e][0] * 3 + kObjEntry[e][1];
    const float r = K[ij] - float(t[e]);
    v += r * r;
    dK[ij] = 2.f * r;
  }
  return v - 1e-4f;
}

struct DeviceFields {
  float *rho = nullptr, *rho_f = nullptr, *k = nullptr, *dk = nullptr, *wsum = nullptr, *g_k = nullptr,
        *g_rho = nullptr, *dvdx = nullptr;
  ~DeviceFields() {
    for (float* p : {rho, rho_f, k, dk, wsum, g_k, g_rho, dvdx})
      if (p) cudaFree(p);
  }
};

__global__ void k_fill(size_t n, float v, float* out) {
  const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) out[i] = v;
}

std::string path_of(const char* prefix, const std::string& name) { return std::string(prefix) + name; }

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace
}  // namespace otm

using namespace otm;

extern "C" {

otm_status otm_driver_config_init(otm_driver_config* cfg) {
  if (!cfg) return OTM_ERR_INVALID_ARGUMENT;
  std::memset(cfg, 0, sizeof(*cfg));
  // HomoConfig::init (cmdline.cpp:4-35)
  cfg->reso = 128;
  cfg->sym = OTM_SYM_NONE;
  cfg->winit = OTM_INIT_IWP;
  cfg->model = OTM_MODEL_OC;
  cfg->vol_ratio = 0.3;
  cfg->heat_ratio[0] = 1.0;
  cfg->heat_ratio[1] = 0.0;
  cfg->finthres = 5e-4;
  cfg->fem_rel_thres = 0.01;
  const double tt[6] = {0.3, 0.2, 0.1, 0.0, 0.0, 0.0};
  for (int i = 0; i < 6; i++) cfg->target_tensor[i] = tt[i];
  cfg->max_iter = 500;
  cfg->init_period = 10;
  return OTM_OK;
}

// ---- ConvergeChecker (Framework.cuh:312-345) ----
void otm_converge_checker_init(otm_converge_checker* c, double thres) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->thres = thres;
}

int otm_converge_checker_step(otm_converge_checker* c, int iter, double obj) {
  if (!c) return 0;
  const int eid = cir_id(iter);
  c->p = eid;
  c->obj[eid] = obj;
  if (iter <= 11) return 0;
  bool out = false;  // the change ratio is above the threshold in one of the last 3 steps
  for (int i = 0; i < 3; i++) {
    const double a = c->obj[cir_id(c->p - i)], b = c->obj[cir_id(c->p - i - 1)];
    out = out || std::fabs(a - b) / std::fabs(b) > c->thres;
  }
  return !out;
}

// ---- VolumeGovernor (Framework.cuh:347-411) ----
void otm_volume_governor_init(otm_volume_governor* g) {
  if (!g) return;
  std::memset(g, 0, sizeof(*g));
  g->volume_bound = 1.0f;
  g->decrease_factor = 1.0f;
  g->val_last = 1.0f;
}

int otm_volume_governor_check(otm_volume_governor* g, float value, float low_bound, float volfrac, int itn) {
  if (!g) return 0;
  g->low_bound = low_bound;
  // small enough objective, or a push at iteration 100
  if (value + 0.0001 < 1e-4 || itn == 100) {
    gov_shrink(g);
    if (g->decrease_factor <= 0.05) return 1;
    g->count = 0;
  }
  const bool reach = std::fabs(g->volume_bound - volfrac) < 1e-2;
  // anti vibration
  if (g->vibrate * (g->val_last - value) < 0)
    g->vibrate_count++;
  else
    g->vibrate_count = 0;
  if (g->vibrate_count >= 8) {
    if (reach) {
      gov_expand(g);
      g->vibrate_count = 0;
    } else {
      gov_shrink(g);
    }
  }
  g->vibrate = g->val_last - value;
  // little progress, large objective and the bound reached
  if (g->val_last - value < 1e-4 && value > 1e-4 && reach)
    g->count++;
  else
    g->count = 0;
  if (g->count >= 5) {
    g->volume_bound += 0.3 * g->decrease * g->decrease_factor;
    g->count = 0;
  }
  g->val_last = value;
  return 0;
}

float otm_volume_governor_decrease(const otm_volume_governor* g) { return g ? g->decrease_factor * g->decrease : 0.f; }

// ---- file formats ----
otm_status otm_write_density_binary(const char* path, const int reso[3], const float* rho_host) {
  if (!path || !reso || !rho_host) return OTM_ERR_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error(std::string("cannot open ") + path);
    return OTM_ERR_INVALID_ARGUMENT;
  }
  const int32_t r[3] = {reso[0], reso[1], reso[2]};
  const size_t n = size_t(reso[0]) * reso[1] * reso[2];
  const bool ok = std::fwrite(r, sizeof(r), 1, f) == 1 && std::fwrite(rho_host, sizeof(float), n, f) == n;
  std::fclose(f);
  if (!ok) {
    set_error(std::string("short write to ") + path);
    return OTM_ERR_INVALID_ARGUMENT;
  }
  return OTM_OK;
}

otm_status otm_read_density_binary(const char* path, int reso[3], float* rho_host, size_t capacity) {
  if (!path || !reso) return OTM_ERR_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error(std::string("cannot open ") + path);
    return OTM_ERR_INVALID_ARGUMENT;
  }
  int32_t r[3] = {0, 0, 0};
  otm_status st = OTM_OK;
  if (std::fread(r, sizeof(r), 1, f) != 1 || r[0] < 1 || r[1] < 1 || r[2] < 1 || r[0] > 1024 || r[1] > 1024 ||
      r[2] > 1024) {
    set_error("density file header is not three sizes in 1..1024");
    st = OTM_ERR_INVALID_ARGUMENT;
  }
  if (st == OTM_OK) {
    for (int i = 0; i < 3; i++) reso[i] = r[i];
    const size_t n = size_t(r[0]) * r[1] * r[2];
    if (rho_host) {
      if (capacity < n) {
        set_error("density buffer smaller than the file's cell count");
        st = OTM_ERR_INVALID_ARGUMENT;
      } else if (std::fread(rho_host, sizeof(float), n, f) != n) {
        set_error("density file is shorter than its header says");
        st = OTM_ERR_INVALID_ARGUMENT;
      }
    }
  }
  std::fclose(f);
  return st;
}

otm_status otm_write_vectors(const char* path, int n_vec, size_t len, const float* const* vecs) {
  if (!path || n_vec < 1 || (len && !vecs)) return OTM_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < n_vec; i++)
    if (len && !vecs[i]) return OTM_ERR_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error(std::string("cannot open ") + path);
    return OTM_ERR_INVALID_ARGUMENT;
  }
  std::vector<float> rec(size_t(n_vec) * len);
  for (size_t j = 0; j < len; j++)
    for (int i = 0; i < n_vec; i++) rec[j * n_vec + i] = vecs[i][j];
  const bool ok = rec.empty() || std::fwrite(rec.data(), sizeof(float), rec.size(), f) == rec.size();
  std::fclose(f);
  if (!ok) {
    set_error(std::string("short write to ") + path);
    return OTM_ERR_INVALID_ARGUMENT;
  }
  return OTM_OK;
}

otm_status otm_read_vectors(const char* path, int n_vec, size_t* len, float* const* vecs, size_t capacity) {
  if (!path || n_vec < 1 || !len) return OTM_ERR_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error(std::string("cannot open ") + path);
    return OTM_ERR_INVALID_ARGUMENT;
  }
  std::fseek(f, 0, SEEK_END);
  const long bytes = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  const size_t nrec = bytes > 0 ? size_t(bytes) / (size_t(n_vec) * sizeof(float)) : 0;
  *len = nrec;
  otm_status st = OTM_OK;
  if (vecs) {
    const size_t take = std::min(nrec, capacity);
    std::vector<float> rec(size_t(n_vec) * take);
    if (!rec.empty() && std::fread(rec.data(), sizeof(float), rec.size(), f) != rec.size()) {
      set_error(std::string("short read from ") + path);
      st = OTM_ERR_INVALID_ARGUMENT;
    } else {
      for (size_t j = 0; j < take; j++)
        for (int i = 0; i < n_vec; i++) vecs[i][j] = rec[j * n_vec + i];
    }
  }
  std::fclose(f);
  return st;
}

otm_status otm_write_heat_matrix(const char* path, const float K[9], int text) {
  if (!path || !K) return OTM_ERR_INVALID_ARGUMENT;
  FILE* f = std::fopen(path, text ? "w" : "wb");
  if (!f) {
    set_error(std::string("cannot open ") + path);
    return OTM_ERR_INVALID_ARGUMENT;
  }
  bool ok = true;
  if (text) {
    for (int i = 0; i < 3 && ok; i++) ok = std::fprintf(f, "%g  %g  %g  \n", K[3 * i], K[3 * i + 1], K[3 * i + 2]) > 0;
  } else {
    ok = std::fwrite(K, sizeof(float), 9, f) == 9;
  }
  std::fclose(f);
  return ok ? OTM_OK : OTM_ERR_INVALID_ARGUMENT;
}

// ---- runCustom (Framework.cu:147-244) ----
otm_status otm_run_custom(const otm_driver_config* cfg, const float* rho0_host, float* rho_out_host,
                          double* obj_history, otm_driver_result* result) {
  if (!cfg || cfg->reso < 8 || cfg->reso > 1024 || cfg->max_iter < 0 ||
      (cfg->model != OTM_MODEL_OC && cfg->model != OTM_MODEL_MMA))
    return OTM_ERR_INVALID_ARGUMENT;
  const int n = cfg->reso;
  const int reso[3] = {n, n, n};
  const size_t ne = size_t(n) * n * n;
  const double t_start = now_s();
  otm_driver_result res;
  std::memset(&res, 0, sizeof(res));

  cudaStream_t s = nullptr;
  OTM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  } guard{s};
  DeviceFields F;
  for (float** p : {&F.rho, &F.rho_f, &F.k, &F.dk, &F.wsum, &F.g_k, &F.g_rho})
    OTM_CUDA(cudaMalloc((void**)p, ne * sizeof(float)));

  // Homogenization_H hom_H(config) with the run's solve tolerance
  otm_config hc;
  otm_config_init(&hc);
  for (int i = 0; i < 3; i++) hc.reso[i] = n;
  hc.fem_rel_thres = cfg->fem_rel_thres;
  otm_homo* homo = nullptr;
  OTM_TRY(otm_homo_create(&hc, &homo));
  struct HomoGuard {
    otm_homo* h;
    ~HomoGuard() { otm_homo_destroy(h); }
  } hg{homo};
  OTM_TRY(otm_homo_set_stream(homo, s));

  // initial density
  const int randtri = cfg->winit == OTM_INIT_RANDOM || cfg->winit == OTM_INIT_RANDCENTER ||
                     cfg->winit == OTM_INIT_REP_RANDCENTER;
  if (rho0_host) {
    OTM_CUDA(cudaMemcpyAsync(F.rho, rho0_host, ne * sizeof(float), cudaMemcpyHostToDevice, s));
  } else {
    std::vector<float> coeffs(randtri ? otm_randtri_coeff_count(cfg->init_period, cfg->winit != OTM_INIT_RANDOM) : 0);
    OTM_TRY(otm_init_density(cfg, F.rho, n, randtri ? coeffs.data() : nullptr, s));
    if (cfg->output_prefix && randtri) {
      const float* v = coeffs.data();
      OTM_TRY(otm_write_vectors(path_of(cfg->output_prefix, "coeff").c_str(), 1, coeffs.size(), &v));
    }
  }
  if (cfg->output_prefix) {
    std::vector<float> h(ne);
    OTM_CUDA(cudaMemcpyAsync(h.data(), F.rho, ne * sizeof(float), cudaMemcpyDeviceToHost, s));
    OTM_CUDA(cudaStreamSynchronize(s));
    OTM_TRY(otm_write_density_binary(path_of(cfg->output_prefix, "init_rand").c_str(), reso, h.data()));
  }

  // objective.eval(): k = filter(rho)^3 (k0 - kmin) + kmin, K^H of k (heat_tensor_t::eval,
  // homoExpression.h:89-100)
  float K[9], dK[9];
  auto evaluate = [&](float* val) -> otm_status {
    OTM_TRY(otm_density_forward(reso, F.rho, n, F.rho_f, F.k, F.dk, F.wsum, OTM_WEIGHT_SPLINE4, 1.5f, 0, 3.0f,
                                float(cfg->heat_ratio[0]), float(cfg->heat_ratio[1]), s));
    OTM_TRY(otm_homo_update(homo, F.k, n));
    double C[9];
    const otm_status st = otm_homo_heat_matrix(homo, C);
    if (st != OTM_OK && st != OTM_ERR_NOT_CONVERGED) return st;
    for (int i = 0; i < 9; i++) K[i] = float(C[i]);
    *val = objective(K, cfg->target_tensor, dK);
    return OTM_OK;
  };
  // objective.backward(1): dObj/dK -> sensitivity -> filter adjoint (homoExpression.h:102-115)
  auto backward = [&]() -> otm_status {
    OTM_TRY(otm_homo_sensitivity(homo, dK, F.g_k, n, 1));
    return otm_density_backward(reso, F.g_k, F.dk, F.wsum, F.g_rho, n, OTM_WEIGHT_SPLINE4, 1.5f, 0, s);
  };

  OTM_CUDA(cudaStreamSynchronize(s));
  const double t_loop = now_s();
  res.init_seconds = t_loop - t_start;
  otm_converge_checker criteria;
  otm_converge_checker_init(&criteria, cfg->finthres);
  FILE* vlog = cfg->output_prefix ? std::fopen(path_of(cfg->output_prefix, "oc_v_log.txt").c_str(), "a") : nullptr;
  struct FileGuard {
    FILE* f;
    ~FileGuard() {
      if (f) std::fclose(f);
    }
  } fg{vlog};
  float val = 0.f;
  if (cfg->model == OTM_MODEL_MMA) {
    // MMAOptimizer mma(1, ne, 1, 0, 1e7, 1); setBound(0.0001, 1) (Framework.cu:174-176)
    otm_mma* mma = nullptr;
    OTM_TRY(otm_mma_create(1, int(ne), 1.0, 0.0, 1e7, 1.0, &mma));
    struct MmaGuard {
      otm_mma* m;
      ~MmaGuard() { otm_mma_destroy(m); }
    } mg{mma};
    OTM_TRY(otm_mma_set_stream(mma, s));
    OTM_TRY(otm_mma_set_bound_scalar(mma, 0.0001f, 1.0f));
    OTM_CUDA(cudaMalloc((void**)&F.dvdx, ne * sizeof(float)));
    k_fill<<<ceil_div(ne, 256), 256, 0, s>>>(ne, float(1.0 / (double(n) * n * n)), F.dvdx);
    count_launches(1);
    for (int itn = 0; itn < cfg->max_iter; itn++) {
      OTM_TRY(evaluate(&val));
      if (obj_history) obj_history[itn] = val;
      res.iterations = itn + 1;
      OTM_TRY(backward());
      if (otm_converge_checker_step(&criteria, itn, val)) {
        res.converged = 1;
        break;
      }
      // minimise the volume subject to objective <= 0: the volume gradient is df0dx and the
      // objective the single constraint (Framework.cu:186-194)
      const float gval = val;
      const float* rows[1] = {F.g_rho};
      OTM_TRY(otm_mma_update(mma, itn, F.rho, F.dvdx, &gval, rows));
      if (vlog) std::fprintf(vlog, "%g %g\n", now_s() - t_start, double(val));
    }
  } else {
    // OCOptimizer oc(ne, 0.001, 0.02, 0.5) with the volume governor (Framework.cu:203-233)
    otm_volume_governor gov;
    otm_volume_governor_init(&gov);
    for (int itn = 0; itn < cfg->max_iter; itn++) {
      OTM_TRY(evaluate(&val));
      if (obj_history) obj_history[itn] = val;
      res.iterations = itn + 1;
      double means[2];  // mean of k (the governor's lower bound) and of rho
      OTM_TRY(field_means(reso, F.k, F.rho, n, s, means));
      otm_volume_governor_check(&gov, val, float(means[0]), float(means[1]), itn);
      OTM_TRY(backward());
      if (otm_converge_checker_step(&criteria, itn, val) && otm_volume_governor_decrease(&gov) < 1e-4) {
        res.converged = 1;
        break;
      }
      OTM_TRY(symmetrize_field(reso, F.rho, n, cfg->sym, 1, s));
      OTM_TRY(symmetrize_field(reso, F.g_rho, n, cfg->sym, 1, s));
      OTM_TRY(otm_oc_filter_sens(F.g_rho, F.rho, size_t(n), reso, 2.0f, s));
      OTM_TRY(otm_oc_update(int(ne), F.g_rho, F.rho, gov.volume_bound, 0.001f, 0.02f, 0.5f, s, nullptr));
    }
    res.volume_bound = gov.volume_bound;
    if (vlog) std::fprintf(vlog, "%g\n", now_s() - t_start);
  }
  OTM_CUDA(cudaStreamSynchronize(s));
  res.loop_seconds = now_s() - t_loop;
  res.objective = val;
  std::memcpy(res.K, K, sizeof(K));
  {
    double means[2];
    OTM_TRY(field_means(reso, F.rho, F.rho, n, s, means));
    res.volume = means[0];
  }
  std::vector<float> out;
  if (rho_out_host || cfg->output_prefix) {
    float* dst = rho_out_host;
    if (!dst) {
      out.resize(ne);
      dst = out.data();
    }
    OTM_CUDA(cudaMemcpyAsync(dst, F.rho, ne * sizeof(float), cudaMemcpyDeviceToHost, s));
    OTM_CUDA(cudaStreamSynchronize(s));
    if (cfg->output_prefix) {
      const std::string name = cfg->model == OTM_MODEL_MMA ? "density_mma" : "density" + std::to_string(n);
      OTM_TRY(otm_write_density_binary(path_of(cfg->output_prefix, name).c_str(), reso, dst));
    }
  }
  OTM_CUDA(cudaStreamSynchronize(s));
  if (result) *result = res;
  return OTM_OK;
}

}  // extern "C"
