// otm_template.cpp -- host-side template matrices of the trilinear heat element.
//
// Same procedure as initTemplateMatrix_H (homogenization/templateMatrix.cpp:21-87): 3x3x3
// Gauss quadrature of B^T B over a cube of half-length a, the node reordering
// mapping = {1,3,2,0,5,7,6,4} to lexicographic local order (i = x + 2y + 4z), and the element
// macro field disp solving KE[1:7,1:7] d = feMu[1:7] with node 0 fixed. Computed in FP64.
#include "otm_template.h"

#include <cmath>
#include <cstring>

namespace otm {

namespace {

void solve_dense(int n, double* A, double* b) {
  for (int k = 0; k < n; k++) {
    int p = k;
    for (int i = k + 1; i < n; i++)
      if (std::fabs(A[i * n + k]) > std::fabs(A[p * n + k])) p = i;
    if (p != k) {
      for (int j = 0; j < n; j++) std::swap(A[k * n + j], A[p * n + j]);
      std::swap(b[k], b[p]);
    }
    for (int i = k + 1; i < n; i++) {
      const double l = A[i * n + k] / A[k * n + k];
      for (int j = k; j < n; j++) A[i * n + j] -= l * A[k * n + j];
      b[i] -= l * b[k];
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = b[i];
    for (int j = i + 1; j < n; j++) s -= A[i * n + j] * b[j];
    b[i] = s / A[i * n + i];
  }
}

// Derivatives of the 8 trilinear shape functions (standard hexahedron order) at (x,y,z).
void shape_derivatives(double x, double y, double z, double q[3][8]) {
  const double sx[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
  const double sy[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
  const double sz[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
  for (int i = 0; i < 8; i++) {
    q[0][i] = sx[i] * (1 + sy[i] * y) * (1 + sz[i] * z) / 8.0;
    q[1][i] = sy[i] * (1 + sx[i] * x) * (1 + sz[i] * z) / 8.0;
    q[2][i] = sz[i] * (1 + sx[i] * x) * (1 + sy[i] * y) / 8.0;
  }
}

}  // namespace

void template_matrices(double a, TemplateMatrices* t) {
  const double gp[3] = {-std::sqrt(0.6), 0.0, std::sqrt(0.6)};
  const double gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  double K[8][8] = {}, F[8][3] = {};
  for (int ii = 0; ii < 3; ii++)
    for (int jj = 0; jj < 3; jj++)
      for (int kk = 0; kk < 3; kk++) {
        double q[3][8];
        shape_derivatives(gp[ii], gp[jj], gp[kk], q);
        // the element is an axis-aligned cube of half-length a: J = a I, B = q / a
        const double w = a * a * a * gw[ii] * gw[jj] * gw[kk];
        for (int i = 0; i < 8; i++) {
          for (int j = 0; j < 8; j++)
            K[i][j] += w * (q[0][i] * q[0][j] + q[1][i] * q[1][j] + q[2][i] * q[2][j]) / (a * a);
          for (int c = 0; c < 3; c++) F[i][c] += w * q[c][i] / a;
        }
      }
  const int mapping[8] = {1, 3, 2, 0, 5, 7, 6, 4};
  for (int i = 0; i < 8; i++) {
    for (int j = 0; j < 8; j++) t->KE[mapping[i]][mapping[j]] = K[i][j];
    for (int c = 0; c < 3; c++) t->feMu[mapping[i]][c] = F[i][c];
  }
  for (int c = 0; c < 3; c++) {
    double A[49], b[7];
    for (int i = 0; i < 7; i++) {
      for (int j = 0; j < 7; j++) A[i * 7 + j] = t->KE[i + 1][j + 1];
      b[i] = t->feMu[i + 1][c];
    }
    solve_dense(7, A, b);
    t->disp[0][c] = 0.0;
    for (int i = 0; i < 7; i++) t->disp[i + 1][c] = b[i];
  }
  // entries by Hamming distance between local nodes
  for (int h = 0; h < 4; h++) t->c[h] = 0.0;
  int cnt[4] = {0, 0, 0, 0};
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) {
      const int h = __builtin_popcount(unsigned(i ^ j));
      t->c[h] += t->KE[i][j];
      cnt[h]++;
    }
  for (int h = 0; h < 4; h++) t->c[h] /= cnt[h];
  double dev = 0.0;
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) dev = std::fmax(dev, std::fabs(t->KE[i][j] - t->c[__builtin_popcount(unsigned(i ^ j))]));
  t->structure_error = dev / std::fabs(t->c[0]);
  // the edge-neighbour entry is zero for the cube element; drop quadrature round-off
  t->face_zero = std::fabs(t->c[1]) <= 1e-12 * std::fabs(t->c[0]);
  if (t->face_zero) t->c[1] = 0.0;
}

void galerkin_level1_table(const TemplateMatrices& t, float* table) {
  auto p1 = [](int r) { return r >= -1 && r <= 1 ? 1.0 - 0.5 * std::abs(r) : 0.0; };
  for (int ez = 0; ez < 4; ez++)
    for (int ey = 0; ey < 4; ey++)
      for (int ex = 0; ex < 4; ex++) {
        const int e = ex + 4 * ey + 16 * ez;
        double a[8];
        int r[8][3];
        for (int i = 0; i < 8; i++) {
          r[i][0] = ex - 2 + (i & 1);
          r[i][1] = ey - 2 + ((i >> 1) & 1);
          r[i][2] = ez - 2 + (i >> 2);
          a[i] = p1(r[i][0]) * p1(r[i][1]) * p1(r[i][2]);
        }
        double Ka[8];
        for (int j = 0; j < 8; j++) {
          double s = 0.0;
          for (int i = 0; i < 8; i++) s += a[i] * t.KE[i][j];
          Ka[j] = s;
        }
        for (int O = 0; O < 27; O++) {
          const int Ox = O % 3 - 1, Oy = (O / 3) % 3 - 1, Oz = O / 9 - 1;
          double s = 0.0;
          for (int j = 0; j < 8; j++)
            s += Ka[j] * p1(r[j][0] - 2 * Ox) * p1(r[j][1] - 2 * Oy) * p1(r[j][2] - 2 * Oz);
          table[e * 27 + O] = float(s);
        }
      }
}

}  // namespace otm
