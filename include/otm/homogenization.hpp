// otm/homogenization.hpp -- header-only C++ drop-in for the reference's host classes, built on
// the C ABI of libopentm_b200.so. Class names, constructor arguments and method signatures
// follow the reference so existing callers compile unchanged:
//   homo::Homogenization_H   homogenization/homogenization.h:15-30
//   homo::MG_H, MGConfig     homogenization/MG.h:8-32
//   homo::Grid_H (subset)    homogenization/grid.h:104-421
//   homo::heat_tensor_t      homogenization/homoExpression.h:69-150, over homo::DensityChain, the
//                            density expression rho.conv(ker).pow(p) * (k0 - kmin) + kmin that
//                            runCustom builds (Framework.cu:163)
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

#include <array>
#include <cstdio>
#include <fstream>
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
    opt_ = opt;
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

  // Not in the reference: heatMatrix(C) and Sensitivity(dC, sens, pitchT, lexiOrder) in one
  // element pass, for a dC that does not depend on C (a linear objective).
  void heatMatrix(double C[3][3], float dC[3][3], float* sens, int pitchT, bool lexiOrder = false) {
    double c[9];
    otm_status s = otm_homo_heat_matrix_sensitivity(h_, c, &dC[0][0], sens, pitchT, lexiOrder ? 1 : 0);
    if (s == OTM_ERR_NOT_CONVERGED)
      std::printf("\033[31mFailed to converge\033[0m\n");
    else
      check(s, "Homogenization_H::heatMatrix");
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) C[i][j] = c[i * 3 + j];
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
  const SolverOptions& options() const { return opt_; }

  float power_penal = 1;
  float diag_strength = 1e6;
  cfg::HomoConfig config;

 private:
  otm_homo* h_ = nullptr;
  SolverOptions opt_;
  float* last_rho_ = nullptr;
  int last_pitch_ = -1;
};

// MGConfig (homogenization/MG.h:8-12).
struct MGConfig {
  int reso[3] = {128, 128, 128};
  bool enableManagedMem = true;
  std::string namePrefix;
};

// One level of the hierarchy (homogenization/grid.h:104-421): its sizes and neighbours. The
// level's vectors live inside the library's handle; the root grid's right-hand sides and
// correction (3 load cases, case-major, x fastest) are device buffers owned by the MG_H view, so
// that v_cycle() works on them as the reference's does on f_g / u_g.
struct Grid_H {
  Grid_H* fine = nullptr;
  Grid_H* Coarse = nullptr;
  bool is_root = false;
  bool assemb_otf = false;  // matrix-free (the fine level)
  std::array<int, 3> cellReso = {};
  int smoother = 0;  // otm_smoother of the level, -1 when it is solved in one direct / cluster launch
  float* f_g[3] = {nullptr, nullptr, nullptr};
  float* u_g[3] = {nullptr, nullptr, nullptr};
  int n_cells(void) const { return cellReso[0] * cellReso[1] * cellReso[2]; }
  std::string getName(void) const {
    return "Grid_" + std::to_string(cellReso[0]) + "x" + std::to_string(cellReso[1]) + "x" +
           std::to_string(cellReso[2]);
  }
  float* getDisplacement(void) { return u_g[0]; }
};

// MG_H (homogenization/MG.h:14-32) as a view of a Homogenization_H, whose handle holds the
// hierarchy.
struct MG_H {
  explicit MG_H(Homogenization_H& hom) : hom_(hom) { sync_grids(); }
  MG_H(const MG_H&) = delete;
  MG_H& operator=(const MG_H&) = delete;
  ~MG_H() { free_root(); }

  std::vector<std::shared_ptr<Grid_H>> grids;  // fine to coarse
  MGConfig mgConfig;

  std::shared_ptr<Grid_H> getRootGrid(void) { return grids.empty() ? nullptr : grids[0]; }

  // build(MGConfig) (MG.cpp:13-44): rebuild the hierarchy for the configuration's resolution.
  void build(MGConfig config) {
    mgConfig = config;
    cfg::HomoConfig hc = hom_.config;
    for (int i = 0; i < 3; i++) hc.reso[i] = config.reso[i];
    hom_.build(hc, hom_.options());
    sync_grids();
  }

  // v_cycle(w_SOR, pre, post) (MG.cpp:46-71): one V-cycle on the root grid's f_g, correction into
  // its u_g. Needs the hierarchy's operators, i.e. a Homogenization_H::update() first.
  void v_cycle(float w_SOR = 1.f, int pre = 1, int post = 1) {
    if (w_SOR != 1.f) throw Error(OTM_ERR_UNSUPPORTED, "MG_H::v_cycle: the smoother is Gauss-Seidel (w_SOR = 1)");
    check(otm_homo_v_cycle(hom_.handle(), root_f_, root_u_, pre, post), "MG_H::v_cycle");
    cudaDeviceSynchronize();
  }

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
  void free_root() {
    if (root_f_) cudaFree(root_f_);
    if (root_u_) cudaFree(root_u_);
    root_f_ = root_u_ = nullptr;
  }
  void sync_grids() {
    grids.clear();
    free_root();
    otm_level_info info;
    check(otm_homo_level(hom_.handle(), 0, &info), "MG_H::grids");
    for (int l = 0; l < info.levels; l++) {
      otm_level_info li;
      check(otm_homo_level(hom_.handle(), l, &li), "MG_H::grids");
      auto g = std::make_shared<Grid_H>();
      g->is_root = (l == 0);
      g->assemb_otf = !li.stencil;
      g->cellReso = {li.reso[0], li.reso[1], li.reso[2]};
      g->smoother = li.smoother;
      grids.push_back(g);
    }
    for (size_t l = 0; l < grids.size(); l++) {
      if (l > 0) grids[l]->fine = grids[l - 1].get();
      if (l + 1 < grids.size()) grids[l]->Coarse = grids[l + 1].get();
    }
    const size_t nv = size_t(grids[0]->n_cells());
    if (cudaMalloc(&root_f_, 3 * nv * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&root_u_, 3 * nv * sizeof(float)) != cudaSuccess)
      throw Error(OTM_ERR_OUT_OF_MEMORY, "MG_H: root grid vectors");
    cudaMemset(root_f_, 0, 3 * nv * sizeof(float));
    cudaMemset(root_u_, 0, 3 * nv * sizeof(float));
    for (int c = 0; c < 3; c++) {
      grids[0]->f_g[c] = root_f_ + c * nv;
      grids[0]->u_g[c] = root_u_ + c * nv;
    }
  }
  Homogenization_H& hom_;
  float* root_f_ = nullptr;
  float* root_u_ = nullptr;
};

// The density expression of runCustom (Framework.cu:163): rho.conv(ker).pow(p) * (k0 - kmin) + kmin
// (the filter of AutoDiff/TensorExpression.h:1095-1185, pow_umker_t :816-843, the affine map), as
// a value type with the interface heat_tensor_t uses: eval(), value(), diff(), backward(diff()).
// rho is the caller's device field (x fastest, element (x,y,z) at x + (y + z*ny)*rho_pitchT);
// grad() receives d objective / d rho after backward(), with the same pitch.
struct DensityChain {
  struct View {
    int pitchT;
    int getPitchT() const { return pitchT; }
  };
  struct TensorRef {
    float* ptr;
    int pitchT;
    float* data() const { return ptr; }
    View view() const { return View{pitchT}; }
  };

  DensityChain(const int reso[3], float* rho, int rho_pitchT, float* grad_rho, float radius = 2.f,
               int weight = OTM_WEIGHT_LINEAR, bool periodic = true, float p = 3.f, float k0 = 1.f, float kmin = 1e-3f)
      : rho_(rho), grad_(grad_rho), pitch_(rho_pitchT > 0 ? rho_pitchT : reso[0]), radius_(radius), weight_(weight),
        periodic_(periodic), p_(p), k0_(k0), kmin_(kmin) {
    for (int i = 0; i < 3; i++) reso_[i] = reso[i];
    const size_t ne = size_t(reso[0]) * reso[1] * reso[2];
    float* bufs[5];
    for (auto& b : bufs)
      if (cudaMalloc(&b, ne * sizeof(float)) != cudaSuccess) throw Error(OTM_ERR_OUT_OF_MEMORY, "DensityChain");
    rho_f_ = bufs[0], k_ = bufs[1], dk_ = bufs[2], wsum_ = bufs[3], diff_ = bufs[4];
  }
  DensityChain(const DensityChain&) = delete;
  DensityChain& operator=(const DensityChain&) = delete;
  ~DensityChain() {
    for (float* b : {rho_f_, k_, dk_, wsum_, diff_}) cudaFree(b);
  }

  void eval() {
    check(otm_density_forward(reso_, rho_, pitch_, rho_f_, k_, dk_, wsum_, weight_, radius_, periodic_ ? 1 : 0, p_,
                              k0_, kmin_, nullptr),
          "DensityChain::eval");
  }
  TensorRef value() { return TensorRef{k_, reso_[0]}; }  // the conductivity field k
  TensorRef diff() { return TensorRef{diff_, reso_[0]}; }  // d objective / d k (written by Sensitivity)
  // chain rule back to rho: grad = filter^T(diff * dk/drho_f)
  void backward(TensorRef g) {
    check(otm_density_backward(reso_, g.data(), dk_, wsum_, grad_, pitch_, weight_, radius_, periodic_ ? 1 : 0,
                               nullptr),
          "DensityChain::backward");
  }
  float* grad() { return grad_; }

 private:
  int reso_[3];
  float* rho_;
  float* grad_;
  int pitch_;
  float radius_;
  int weight_;
  bool periodic_;
  float p_, k0_, kmin_;
  float *rho_f_ = nullptr, *k_ = nullptr, *dk_ = nullptr, *wsum_ = nullptr, *diff_ = nullptr;
};

// Reference counting of the expression graph (each user's eval counts once; backward runs when
// every user has propagated its gradient).
struct RefCounter {
  int n_eval = 0, n_backward = 0;
  void c_eval() { n_eval++; }
  void c_backward() { n_backward++; }
  bool finishedBackward() const { return n_backward >= n_eval; }
  void reset() { n_eval = n_backward = 0; }
};

// heat_tensor_t (homogenization/homoExpression.h:69-150): eval() evaluates the density expression,
// updates the homogenization domain with it and stores K^H in H_; the caller writes the gradient
// of its objective with respect to K^H into gradH_ (the reference's scalar autodiff does that
// through operator()(i, j)); backward() turns it into the element sensitivity (Sensitivity,
// pitched lexicographic) and back-propagates it through the density expression.
template <typename Scalar, typename DensityExp_t>
struct heat_tensor_t {
  Scalar H_[3][3] = {};
  Scalar gradH_[3][3] = {};
  DensityExp_t& densityField;
  RefCounter counter;
  Homogenization_H& domain_;
  bool hold_on = false;
  bool expired = true;

  heat_tensor_t(Homogenization_H& dom, DensityExp_t& rho) : densityField(rho), domain_(dom), expired(true) {}

  Scalar& value(int i, int j) { return H_[i][j]; }
  Scalar& grad(int i, int j) { return gradH_[i][j]; }
  void reset(void) { counter.reset(); }
  void holdOn(void) { hold_on = true; }
  void holdOff(void) { hold_on = false; }

  void eval(void) {
    counter.c_eval();
    if (expired && !hold_on) {
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) gradH_[i][j] = 0;
      densityField.eval();
      domain_.update(densityField.value().data(), densityField.value().view().getPitchT());
      domain_.heatMatrix(H_);
      expired = false;
    }
    if (hold_on)
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) gradH_[i][j] = 0;
  }

  void backward() {
    counter.c_backward();
    if (counter.finishedBackward() && (!expired || hold_on)) {
      expired = true;
      counter.reset();
      float g[3][3];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) g[i][j] = float(gradH_[i][j]);
      domain_.Sensitivity(g, densityField.diff().data(), densityField.diff().view().getPitchT(), true);
      densityField.backward(densityField.diff());
    }
  }

  void writeTo(const std::string& filename) {
    std::ofstream ofs(filename, std::ios::binary);
    ofs.write((const char*)(&H_[0][0]), sizeof(H_));
  }
  void writeToTxt(const std::string& filename) {
    std::ofstream ofs(filename);
    for (int i = 0; i < 3; i++) {
      for (int j = 0; j < 3; j++) ofs << H_[i][j] << "  ";
      ofs << "\n";
    }
  }
  const Scalar* data(void) { return &H_[0][0]; }
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
