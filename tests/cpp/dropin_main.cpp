// Drop-in check of the C++ wrapper: the reference's call sequence (Homogenization_H::update,
// heatMatrix, Sensitivity; OCOptimizer::filterSens/update; MMAOptimizer::update; mmasubDevice)
// compiled unchanged against include/otm/homogenization.hpp, then runCustom / ConvergeChecker /
// VolumeGovernor of the driver layer, heat_tensor_t's eval / backward over the density chain, and
// MG_H's grids and v_cycle. Prints K^H and checksums; the
// pytest driver compares them with the Python path.
#include <cmath>
#include <cstdio>
#include <vector>

#include "otm/homogenization.hpp"

static float u01(unsigned long long i) {
  unsigned long long z = i + 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return float((z >> 11) * (1.0 / 9007199254740992.0));
}

int main() {
  const int n = 16, ne = n * n * n, pitchT = 32;
  cfg::HomoConfig config;
  config.init();
  config.reso[0] = config.reso[1] = config.reso[2] = n;
  config.femRelThres = 1e-6;
  homo::SolverOptions opt;
  opt.pre_smooth = opt.post_smooth = 2;
  homo::Homogenization_H hom(config, opt);

  std::vector<float> h(size_t(n) * n * pitchT, 0.f);
  for (int e = 0; e < ne; e++) {
    const float rho = 0.001f + 0.999f * u01(e);
    h[size_t(e / n) * pitchT + e % n] = 1e-3f + rho * rho * rho * (1.f - 1e-3f);
  }
  float *rho_d = nullptr, *sens_d = nullptr;
  cudaMalloc(&rho_d, h.size() * sizeof(float));
  cudaMalloc(&sens_d, h.size() * sizeof(float));
  cudaMemcpy(rho_d, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice);

  hom.update(rho_d, pitchT);
  double C[3][3];
  hom.heatMatrix(C);
  float dC[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  hom.Sensitivity(dC, sens_d, pitchT, true);
  std::vector<float> s(h.size());
  cudaMemcpy(s.data(), sens_d, s.size() * sizeof(float), cudaMemcpyDeviceToHost);
  double ssum = 0;
  for (float v : s) ssum += v;
  std::printf("C %.9e %.9e %.9e %.9e %.9e %.9e\n", C[0][0], C[0][1], C[0][2], C[1][1], C[1][2], C[2][2]);
  std::printf("sens_sum %.9e\n", ssum);
  {
    // K^H and the sensitivity in one element pass (a handle of its own, the same field)
    homo::Homogenization_H hom2(config, opt);
    hom2.update(rho_d, pitchT);
    double C2[3][3];
    hom2.heatMatrix(C2, dC, sens_d, pitchT, true);
    std::vector<float> s2(h.size());
    cudaMemcpy(s2.data(), sens_d, s2.size() * sizeof(float), cudaMemcpyDeviceToHost);
    bool same = true;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) same = same && C2[i][j] == C[i][j];
    for (size_t i = 0; i < s.size(); i++) same = same && s2[i] == s[i];
    std::printf("fused_same %d\n", int(same));
  }

  // MG_H view: re-solve from zero with a tighter tolerance
  homo::MG_H mg(hom);
  double rr = mg.solveEquation(1e-7, false);
  std::printf("relres %.3e\n", rr);

  // OC on the unpitched sensitivity of -trace(K^H)
  float *srho = nullptr, *ss = nullptr;
  cudaMalloc(&srho, ne * sizeof(float));
  cudaMalloc(&ss, ne * sizeof(float));
  std::vector<float> r0(ne, 0.3f), g(ne);
  for (int e = 0; e < ne; e++) g[e] = -(0.1f + u01(ne + e));
  cudaMemcpy(srho, r0.data(), ne * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(ss, g.data(), ne * sizeof(float), cudaMemcpyHostToDevice);
  homo::OCOptimizer oc(ne, 0.001f, 0.2f, 0.5f);
  int reso[3] = {n, n, n};
  oc.filterSens(ss, srho, n, reso, 2.0f);
  oc.update(ss, srho, 0.25f);
  cudaMemcpy(r0.data(), srho, ne * sizeof(float), cudaMemcpyDeviceToHost);
  double vol = 0;
  for (float v : r0) vol += v;
  std::printf("oc_vol %.6f\n", vol / ne);

  // MMA: minimise sum (x - t)^2 subject to mean(x) <= 0.3 through the float interface
  homo::MMAOptimizer mma(1, ne, 1, 0, 1e3, 1);
  mma.setBound(0.f, 1.f);
  std::vector<float> x(ne, 0.5f), t(ne), df(ne), dg(ne, 1.f / (0.3f * ne));
  for (int e = 0; e < ne; e++) t[e] = u01(3 * ne + e);
  float *xd, *dfd, *dgd;
  cudaMalloc(&xd, ne * sizeof(float));
  cudaMalloc(&dfd, ne * sizeof(float));
  cudaMalloc(&dgd, ne * sizeof(float));
  cudaMemcpy(xd, x.data(), ne * sizeof(float), cudaMemcpyHostToDevice);
  cudaMemcpy(dgd, dg.data(), ne * sizeof(float), cudaMemcpyHostToDevice);
  for (int it = 1; it <= 30; it++) {
    cudaMemcpy(x.data(), xd, ne * sizeof(float), cudaMemcpyDeviceToHost);
    double sx = 0;
    for (int e = 0; e < ne; e++) {
      df[e] = 2.f * (x[e] - t[e]);
      sx += x[e];
    }
    float gval = float(sx / (0.3 * ne) - 1.0);
    cudaMemcpy(dfd, df.data(), ne * sizeof(float), cudaMemcpyHostToDevice);
    float* rows[1] = {dgd};
    mma.update(it, xd, dfd, &gval, rows);
  }
  cudaMemcpy(x.data(), xd, ne * sizeof(float), cudaMemcpyDeviceToHost);
  double mean = 0;
  for (float v : x) mean += v;
  std::printf("mma_mean %.6f\n", mean / ne);
  cudaDeviceSynchronize();
  // the design driver as main.cpp calls it, on a small cell with two iterations
  {
    cfg::HomoConfig dc;
    dc.init();
    dc.reso[0] = dc.reso[1] = dc.reso[2] = 16;
    dc.max_iter = 2;
    dc.heatRatio[1] = 1e-4;
    dc.winit = cfg::InitWay::IWP;
    dc.model = cfg::Model::oc;
    std::vector<float> rho = runCustom(dc);
    double sum = 0;
    for (float v : rho) sum += v;
    std::printf("design_sum %.9e\n", sum);
    ConvergeChecker cc(1e-3);
    VolumeGovernor vg;
    vg.volume_check(-1e-3f, 0.25f, 0.5f, 0);
    std::printf("governor %.7f %d\n", vg.get_volume_bound(), int(cc.is_converge(0, 1.0)));
  }
  // heat_tensor_t over the density chain of runCustom (homoExpression.h:69-150), used as a design
  // step uses it: eval() gives K^H, the objective's gradient goes into gradH_, backward() gives
  // d objective / d rho
  {
    const int reso[3] = {n, n, n};
    std::vector<float> hr(ne);
    for (int e = 0; e < ne; e++) hr[e] = u01(5 * ne + e);
    float *rho_e = nullptr, *grad_e = nullptr;
    cudaMalloc(&rho_e, ne * sizeof(float));
    cudaMalloc(&grad_e, ne * sizeof(float));
    cudaMemcpy(rho_e, hr.data(), ne * sizeof(float), cudaMemcpyHostToDevice);
    homo::Homogenization_H hom2(config, opt);
    homo::DensityChain dens(reso, rho_e, n, grad_e);
    homo::heat_tensor_t<float, homo::DensityChain> Hh(hom2, dens);
    Hh.eval();
    for (int i = 0; i < 3; i++) Hh.gradH_[i][i] = -1.f;  // objective -trace(K^H)
    Hh.backward();
    std::vector<float> g(ne);
    cudaMemcpy(g.data(), dens.grad(), ne * sizeof(float), cudaMemcpyDeviceToHost);
    double gs = 0;
    for (float v : g) gs += v;
    std::printf("ht_C %.9e %.9e %.9e %.9e %.9e %.9e\n", Hh.H_[0][0], Hh.H_[0][1], Hh.H_[0][2], Hh.H_[1][1],
                Hh.H_[1][2], Hh.H_[2][2]);
    std::printf("ht_grad_sum %.9e\n", gs);
    // MG_H: the grids and one V(2,2) cycle on the root grid's right-hand sides
    homo::MG_H mg2(hom2);
    auto root = mg2.getRootGrid();
    std::printf("mg_levels %d %d %d\n", int(mg2.grids.size()), root->cellReso[0], int(root->Coarse != nullptr));
    std::vector<float> fr(3 * size_t(ne));
    for (int i = 0; i < 3 * ne; i++) fr[i] = u01(7 * ne + i) - 0.5f;
    cudaMemcpy(root->f_g[0], fr.data(), fr.size() * sizeof(float), cudaMemcpyHostToDevice);
    mg2.v_cycle(1.f, 2, 2);
    cudaMemcpy(fr.data(), root->u_g[0], fr.size() * sizeof(float), cudaMemcpyDeviceToHost);
    double un = 0;
    for (float v : fr) un += double(v) * v;
    std::printf("vc_norm %.9e\n", std::sqrt(un));
    cudaFree(rho_e);
    cudaFree(grad_e);
  }
  std::printf("ok\n");
  return 0;
}
