// otm/homogenization.hpp -- header-only C++ drop-in for the reference's host classes, built on
// the C ABI of libopentm_b200.so. Class names, constructor arguments and method signatures
// follow the reference so existing callers compile unchanged:
//   homo::Homogenization_H   homogenization/homogenization.h:15-30
//   homo::MG_H (subset)      homogenization/MG.h:14-32
//   homo::OCOptimizer        optimization/OCOptimizer.h:7-20
//   homo::MMAOptimizer       optimization/mmaOptimizer.h:12-35
//   mmasubDevice             optimization/mmaOpt.h:14-19
//   cfg::HomoConfig          cmdline.h:12-33
//   ConvergeChecker, VolumeGovernor   homogenization/Framework.cuh:312-411
//   runCustom                Framework.cu:147-244
//   runInstance, wrapper_homo main.cpp:17-62
// Errors the reference reported with printf/exit/exceptions surface as std::runtime_error
// (homo::Error) carrying the otm_status; a solve that hits the iteration cap prints a
// warning and continues, as MG_H::solveEquation does (homogenization/MG.cpp:392-428).
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>

#include <vector>

#include "opentm_b200.h"
#include "opentm_b200_driver.h"
#include "opentm_b200_mma.h"

namespace cfg {
enum class Objective : uint8_t { bulk, shear, npr, custom };
enum class Symmetry : uint8_t { reflect3, reflect6, rotate3, rotate2, NONE };
enum class InitWay : uint8_t { random, randcenter, noise, manual, interp, rep_randcenter, P, G, D, IWP, example };
enum class Model : uint8_t { mma, oc };

// cmdline.h:12-33; init() sets the defaults of cmdline.cpp:4-35.
struct HomoConfig {
  Symmetry sym = Symmetry::NONE;
  InitWay winit = InitWay::IWP;
  Model model = Model::oc;
  int reso[3] = {128, 128, 128};
  double volRatio = 0.3;
  double heatRatio[2] = {1, 0};
  double finthres = 5e-4;
  double filterRadius = 2.0;
  double designStep = 0.05;
  double dampRatio = 0.5;
  double femRelThres = 0.01;
  double target_tensor[6] = {0.3, 0.2, 0.1, 0, 0, 0};
  std::string outprefix, testname, inputrho = "init rand";
  bool useManagedMemory = true;
  int logrho = 0, logc = 0, logsens = 0, logobj = 0;
  int max_iter = 500;
  int initperiod = 10;
  void init() { *this = HomoConfig(); }
};
}  // namespace cfg

namespace homo {

struct Error : std::runtime_error {
  otm_status status;
  Error(otm_status s, const std::string& where)
      : std::runtime_error(where + ": " + otm_status_string(s) + " (" + otm_last_error() + ")"), status(s) {}
};

inline void check(otm_status s, const char* where) {
  if (s != OTM_OK) throw Error(s, where);
}

// Solver options beyond cfg::HomoConfig (precision form, cycle shape, iteration cap).
struct SolverOptions {
  int pre_smooth = 1, post_smooth = 1;
  int max_iter = 200;
  otm_solver solver = OTM_SOLVER_PCG;
  otm_precision precision = OTM_PRECISION_FP32;
};

struct MG_H;

struct Homogenization_H {
  explicit Homogenization_H(cfg::HomoConfig config, SolverOptions opt = SolverOptions()) { build(config, opt); }
  Homogenization_H(const Homogenization_H&) = delete;
  Homogenization_H& operator=(const Homogenization_H&) = delete;
  ~Homogenization_H() {
    if (h_) otm_homo_destroy(h_);
  }

  void build(cfg::HomoConfig homconfig, SolverOptions opt = SolverOptions()) {
    if (h_) otm_homo_destroy(h_);
    h_ = nullptr;
    config = homconfig;
    otm_config c;
    otm_config_init(&c);
    for (int i = 0; i < 3; i++) c.reso[i] = config.reso[i];
    c.fem_rel_thres = config.femRelThres;
    c.pre_smooth = opt.pre_smooth;
    c.post_smooth = opt.post_smooth;
    c.max_iter = opt.max_iter;
    c.solver = opt.solver;
    c.precision = opt.precision;
    c.power_penal = power_penal;
    check(otm_homo_create(&c, &h_), "Homogenization_H::build");
  }

  // update(float* rho, int pitchT) (homogenization.cpp:76-81); rho == nullptr re-uses the
  // last field, which the caller keeps alive.
  void update(float* rho = nullptr, int pitchT = -1) {
    if (rho) {
      last_rho_ = rho;
      last_pitch_ = pitchT;
    }
    if (!last_rho_) throw Error(OTM_ERR_STATE, "Homogenization_H::update: no density field");
    check(otm_homo_update(h_, last_rho_, last_pitch_), "Homogenization_H::update");
  }

  void heatMatrix(double C[3][3]) {
    double c[9];
    otm_status s = otm_homo_heat_matrix(h_, c);
    if (s == OTM_ERR_NOT_CONVERGED)
      std::printf("\033[31mFailed to converge\033[0m\n");
    else
      check(s, "Homogenization_H::heatMatrix");
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) C[i][j] = c[i * 3 + j];
  }

  void heatMatrix(float C[3][3]) {
    double c[3][3];
    heatMatrix(c);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) C[i][j] = float(c[i][j]);
  }

  void Sensitivity(float dC[3][3], float* sens, int pitchT, bool lexiOrder = false) {
    check(otm_homo_sensitivity(h_, &dC[0][0], sens, pitchT, lexiOrder ? 1 : 0), "Homogenization_H::Sensitivity");
  }

  // The reference stores the strength and never uses it (homogenization.cpp:83-87).
  void ConfigDiagPrecondition(float strength) { diag_strength = strength; }

  void setStream(cudaStream_t s) { check(otm_homo_set_stream(h_, s), "Homogenization_H::setStream"); }
  otm_solve_stats stats() const {
    otm_solve_stats st;
    otm_homo_get_stats(h_, &st);
    return st;
  }
  otm_homo* handle() { return h_; }

  float power_penal = 1;
  float diag_strength = 1e6;
  cfg::HomoConfig config;

 private:
  otm_homo* h_ = nullptr;
  float* last_rho_ = nullptr;
  int last_pitch_ = -1;
};

// MG_H view of a Homogenization_H (homogenization/MG.h:14-32): the hierarchy lives inside the
// handle, so only the solve-level entry points are exposed.
struct MG_H {
  explicit MG_H(Homogenization_H& hom) : hom_(hom) {}
  // solveEquation(tol, with_guess) (MG.cpp:80-142): solves all 3 load cases, returns the
  // largest relative residual.
  double solveEquation(double tol = 1e-2, bool with_guess = true) {
    if (!with_guess) reset_displacement();
    check(otm_homo_set_tolerance(hom_.handle(), tol), "MG_H::solveEquation");
    otm_solve_stats st;
    otm_status s = otm_homo_solve(hom_.handle(), &st);
    if (s == OTM_ERR_NOT_CONVERGED)
      std::printf(" - r_rel = %le\n", st.rel_res[0]);
    else
      check(s, "MG_H::solveEquation");
    double r = 0;
    for (double v : st.rel_res) r = v > r ? v : r;
    return r;
  }
  void reset_displacement() { check(otm_homo_reset_displacement(hom_.handle()), "MG_H::reset_displacement"); }
  void updateStencils() { hom_.update(); }

 private:
  Homogenization_H& hom_;
};

struct OCOptimizer {
  int ne = 0;
  float step_limit = 0.02f;
  float damp = 0.5f;
  float minRho = 0.001f;
  cudaStream_t stream = nullptr;
  OCOptimizer(int Ne, float min_density, float stepLimit, float dampExponent)
      : ne(Ne), step_limit(stepLimit), damp(dampExponent), minRho(min_density) {}
  OCOptimizer(float min_density, float stepLimit, float dampExponent)
      : step_limit(stepLimit), damp(dampExponent), minRho(min_density) {}
  void filterSens(float* sens, const float* rho, size_t pitchT, int reso[3], float radius = 2) {
    check(otm_oc_filter_sens(sens, rho, pitchT, reso, radius, stream), "OCOptimizer::filterSens");
  }
  void update(const float* sens, float* rho, float volratio) {
    check(otm_oc_update(ne, sens, rho, volratio, minRho, step_limit, damp, stream, nullptr), "OCOptimizer::update");
  }
};

class MMAOptimizer {
 public:
  int n, m;
  double a0;
  double a, c, d;
  MMAOptimizer(int nconstrain, int nvar, double a0_, double a_, double c_, double d_)
      : n(nvar), m(nconstrain), a0(a0_), a(a_), c(c_), d(d_) {
    check(otm_mma_create(m, n, a0, a, c, d, &h_), "MMAOptimizer");
  }
  MMAOptimizer(const MMAOptimizer&) = delete;
  MMAOptimizer& operator=(const MMAOptimizer&) = delete;
  ~MMAOptimizer() {
    if (h_) otm_mma_destroy(h_);
  }
  void setBound(float* xmin, float* xmax) { check(otm_mma_set_bound(h_, xmin, xmax), "MMAOptimizer::setBound"); }
  void setBound(float xmin, float xmax) {
    check(otm_mma_set_bound_scalar(h_, xmin, xmax), "MMAOptimizer::setBound");
  }
  void update(int itn, float* x, float* dfdx, float* gval, float** dgdx) {
    check(otm_mma_update(h_, itn, x, dfdx, gval, dgdx), "MMAOptimizer::update");
  }

 private:
  otm_mma* h_ = nullptr;
};

}  // namespace homo

// ---- the driver layer (global names, as in the reference) ----
struct ConvergeChecker {
  ConvergeChecker(double thres_ = 1e-3) { otm_converge_checker_init(&c_, thres_); }
  bool is_converge(int iter, double obj) { return otm_converge_checker_step(&c_, iter, obj) != 0; }

 private:
  otm_converge_checker c_{};
};

struct VolumeGovernor {
  VolumeGovernor() { otm_volume_governor_init(&g_); }
  float get_volume_bound() { return g_.volume_bound; }
  int volume_check(float value, float lowBound, float volfrac, int itn) {
    return otm_volume_governor_check(&g_, value, lowBound, volfrac, itn);
  }
  float get_current_decrease() { return otm_volume_governor_decrease(&g_); }

 private:
  otm_volume_governor g_{};
};

// runCustom (Framework.cu:147-244): the design loop; rho0 (reso^3 values) replaces initDensity.
// Files are written only when config.outprefix is not empty (the reference always writes them,
// with OpenVDB densities; here they are in the binary density format).
inline std::vector<float> runCustom(cfg::HomoConfig config, std::vector<float>* rho0 = nullptr) {
  otm_driver_config c;
  otm_driver_config_init(&c);
  c.reso = config.reso[0];
  c.sym = int(config.sym);
  c.winit = int(config.winit);
  c.model = int(config.model);
  c.vol_ratio = config.volRatio;
  c.heat_ratio[0] = config.heatRatio[0];
  c.heat_ratio[1] = config.heatRatio[1];
  c.finthres = config.finthres;
  c.fem_rel_thres = config.femRelThres;
  for (int i = 0; i < 6; i++) c.target_tensor[i] = config.target_tensor[i];
  c.max_iter = config.max_iter;
  c.init_period = config.initperiod;
  c.input_path = config.inputrho.c_str();
  c.output_prefix = config.outprefix.empty() ? nullptr : config.outprefix.c_str();
  const size_t ne = size_t(c.reso) * c.reso * c.reso;
  if (rho0 && rho0->size() != ne)
    throw homo::Error(OTM_ERR_INVALID_ARGUMENT, "runCustom: rho0 does not hold reso^3 values");
  std::vector<float> rho(ne);
  homo::check(otm_run_custom(&c, rho0 ? rho0->data() : nullptr, rho.data(), nullptr, nullptr), "runCustom");
  return rho;
}

// runInstance / wrapper_homo (main.cpp:17-62)
inline std::vector<float> runInstance(int reso, std::vector<double> heat_ratios, std::vector<double> target_ratio,
                                      cfg::InitWay initway, cfg::Model model) {
  cfg::HomoConfig config;
  config.init();
  config.reso[0] = config.reso[1] = config.reso[2] = reso;
  if (heat_ratios.size() != 2 || target_ratio.size() < 6)
    throw homo::Error(OTM_ERR_INVALID_ARGUMENT, "runInstance: wrong size of heat_ratios or target_ratio");
  for (int i = 0; i < 2; i++) config.heatRatio[i] = heat_ratios[i];
  for (int i = 0; i < 6; i++) config.target_tensor[i] = target_ratio[i];
  config.winit = initway;
  config.model = model;
  return runCustom(config);
}

class wrapper_homo {
  cfg::HomoConfig config;
  std::vector<float> rho;

 public:
  wrapper_homo() { config.init(); }
  void setDensity(std::vector<float> rho_) { rho = rho_; }
  void setConfig(int reso, std::vector<double> heat_ratios, std::vector<double> target_ratio, cfg::Model model) {
    config.init();
    config.reso[0] = config.reso[1] = config.reso[2] = reso;
    if (heat_ratios.size() != 2 || target_ratio.size() < 6)
      throw homo::Error(OTM_ERR_INVALID_ARGUMENT, "setConfig: wrong size of heat_ratios or target_ratio");
    for (int i = 0; i < 2; i++) config.heatRatio[i] = heat_ratios[i];
    for (int i = 0; i < 6; i++) config.target_tensor[i] = target_ratio[i];
    config.model = model;
  }
  std::vector<float> optimize() { return runCustom(config, &rho); }
};

// mmasubDevice (optimization/mmaOpt.h:14-19) with the reference's exact signature.
inline void mmasubDevice(int ncontrain, int nvar, int itn, double* xvar, double* xmin, double* xmax, double* xold1,
                         double* xold2, double f0val, double* df0dx, double* gval, cudaPitchedPtr dgdx, double* low,
                         double* upp, double a0, double* a, double* c, double* d, double move) {
  otm_pitched_ptr p{dgdx.ptr, dgdx.pitch, dgdx.xsize, dgdx.ysize};
  homo::check(otm_mmasub_device(ncontrain, nvar, itn, xvar, xmin, xmax, xold1, xold2, f0val, df0dx, gval, p, low, upp,
                                a0, a, c, d, move, nullptr),
              "mmasubDevice");
}
