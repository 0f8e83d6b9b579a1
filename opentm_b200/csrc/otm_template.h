// otm_template.h -- host-side template matrices of the trilinear heat element.
#pragma once

namespace otm {

struct TemplateMatrices {
  double KE[8][8];    // lexicographic local order i = x + 2y + 4z
  double feMu[8][3];  // element load matrix of the 3 unit gradients (reference convention)
  double disp[8][3];  // element macro field, node 0 fixed
  double c[4];        // KE entry by Hamming distance of the local nodes
  double structure_error;
  bool face_zero;
};

// Element half-length a = 1 / (2 reso_x) (homogenization/homogenization.cpp:211).
void template_matrices(double a, TemplateMatrices* t);

// 64 x 27 table of the level-1 Galerkin operator: A_1(V, V+O) = sum_e k_e table[e*27 + O]
// over the 4^3 fine elements with lower corners 2V - 2 + (ex, ey, ez), e = ex + 4ey + 16ez.
void galerkin_level1_table(const TemplateMatrices& t, float* table);

}  // namespace otm
