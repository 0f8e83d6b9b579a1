// otm_oracle.cpp -- FP64 CPU restatement of OpenTM's thermal homogenization hot path.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product (opentm_b200/) links, loads or calls this
// file. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it, and
// there only as the checker or as the timed CPU baseline.
//
// Parity status: the reference publishes no golden vectors and cannot be built offline
// (Eigen, glm and OpenVDB are absent), so this oracle is pinned by known-answer tests
// derived from the mathematics (rho == 1 gives K^H = I, laminates give the arithmetic and
// harmonic means in closed form, a Jacobi-PCG solve without multigrid cross-checks the
// multigrid path, finite differences check dK^H/dk_e). Direct parity with the reference's
// own outputs is unpinned.
//
// Everything here follows the reference's algorithm; each function cites the reference
// file:line (paths relative to the OpenTM project root) whose behaviour it restates.
// Conventions shared with the CUDA path:
//   * a cell has n[0] x n[1] x n[2] voxels (elements) and as many periodic vertices;
//     index(x, y, z) = x + n0 * (y + n1 * z), x fastest;
//   * element e at (x, y, z) has corner j at (x + (j&1), y + (j>>1&1), z + (j>>2));
//   * the solver conductivity is k_e = 1e-9 + k^p (homogenization/grid.cu:405, grid.h:429);
//   * the 3 load cases use the element macro fields of the template matrix
//     (homogenization/templateMatrix.cpp:74-85), i.e. the reference's axis convention.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double kRhoPenalMin = 1e-9;  // homogenization/grid.h:429

inline int wrap(int a, int n) {
  a %= n;
  return a < 0 ? a + n : a;
}

struct Dims {
  int n[3];
  size_t nv() const { return size_t(n[0]) * n[1] * n[2]; }
  size_t id(int x, int y, int z) const {
    return size_t(wrap(x, n[0])) + size_t(n[0]) * (size_t(wrap(y, n[1])) + size_t(n[1]) * size_t(wrap(z, n[2])));
  }
};

// Dense LU with partial pivoting, solves A x = b in place (A is n x n row-major).
bool lu_solve(int n, std::vector<double> A, double* b) {
  std::vector<int> piv(n);
  for (int k = 0; k < n; k++) {
    int p = k;
    for (int i = k + 1; i < n; i++)
      if (std::fabs(A[i * n + k]) > std::fabs(A[p * n + k])) p = i;
    if (A[p * n + k] == 0.0) return false;
    if (p != k) {
      for (int j = 0; j < n; j++) std::swap(A[k * n + j], A[p * n + j]);
      std::swap(b[k], b[p]);
    }
    for (int i = k + 1; i < n; i++) {
      double l = A[i * n + k] / A[k * n + k];
      for (int j = k; j < n; j++) A[i * n + j] -= l * A[k * n + j];
      b[i] -= l * b[k];
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = b[i];
    for (int j = i + 1; j < n; j++) s -= A[i * n + j] * b[j];
    b[i] = s / A[i * n + i];
  }
  return true;
}

// ---------------------------------------------------------------------------------------
// Template matrices (homogenization/templateMatrix.cpp:21-87).
// ---------------------------------------------------------------------------------------
void template_matrix(double a, double KE[64], double feMu[24], double disp[24]) {
  const double gp[3] = {-std::sqrt(3.0 / 5.0), 0.0, std::sqrt(3.0 / 5.0)};
  const double gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
  // node coordinates of the standard hexahedron, templateMatrix.cpp:55-62
  const double Jr[8][3] = {{-a, -a, -a}, {a, -a, -a}, {a, a, -a}, {-a, a, -a},
                           {-a, -a, a},  {a, -a, a},  {a, a, a},  {-a, a, a}};
  double K[8][8] = {}, F[8][3] = {};
  for (int ii = 0; ii < 3; ii++)
    for (int jj = 0; jj < 3; jj++)
      for (int kk = 0; kk < 3; kk++) {
        double x = gp[ii], y = gp[jj], z = gp[kk];
        // shape function derivatives in natural coordinates, templateMatrix.cpp:40-48
        double q[3][8] = {
            {-((y - 1) * (z - 1)) / 8, ((y - 1) * (z - 1)) / 8, -((y + 1) * (z - 1)) / 8,
             ((y + 1) * (z - 1)) / 8, ((y - 1) * (z + 1)) / 8, -((y - 1) * (z + 1)) / 8,
             ((y + 1) * (z + 1)) / 8, -((y + 1) * (z + 1)) / 8},
            {-((x - 1) * (z - 1)) / 8, ((x + 1) * (z - 1)) / 8, -((x + 1) * (z - 1)) / 8,
             ((x - 1) * (z - 1)) / 8, ((x - 1) * (z + 1)) / 8, -((x + 1) * (z + 1)) / 8,
             ((x + 1) * (z + 1)) / 8, -((x - 1) * (z + 1)) / 8},
            {-((x - 1) * (y - 1)) / 8, ((x + 1) * (y - 1)) / 8, -((x + 1) * (y + 1)) / 8,
             ((x - 1) * (y + 1)) / 8, ((x - 1) * (y - 1)) / 8, -((x + 1) * (y - 1)) / 8,
             ((x + 1) * (y + 1)) / 8, -((x - 1) * (y + 1)) / 8}};
        double J[3][3] = {};
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++)
            for (int t = 0; t < 8; t++) J[r][c] += q[r][t] * Jr[t][c];
        double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        double Ji[3][3] = {
            {(J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det, (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det,
             (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det},
            {(J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det, (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det,
             (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det},
            {(J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det, (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det,
             (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det}};
        double B[3][8] = {};
        for (int r = 0; r < 3; r++)
          for (int t = 0; t < 8; t++)
            for (int c = 0; c < 3; c++) B[r][t] += Ji[r][c] * q[c][t];
        double w = det * gw[ii] * gw[jj] * gw[kk];
        // heat_matrix = identity (he = 1), templateMatrix.cpp:24-26, 66-67
        for (int i = 0; i < 8; i++) {
          for (int j = 0; j < 8; j++) K[i][j] += w * (B[0][i] * B[0][j] + B[1][i] * B[1][j] + B[2][i] * B[2][j]);
          for (int c = 0; c < 3; c++) F[i][c] += w * B[c][i];
        }
      }
  // node reordering, templateMatrix.cpp:74-82
  const int mapping[8] = {1, 3, 2, 0, 5, 7, 6, 4};
  for (int i = 0; i < 8; i++) {
    for (int j = 0; j < 8; j++) KE[mapping[i] * 8 + mapping[j]] = K[i][j];
    for (int c = 0; c < 3; c++) feMu[mapping[i] * 3 + c] = F[i][c];
  }
  // element macro field: KE[1:7,1:7] d = feMu[1:7], node 0 fixed, templateMatrix.cpp:84-85
  for (int c = 0; c < 3; c++) {
    std::vector<double> A(49);
    double b[7];
    for (int i = 0; i < 7; i++) {
      for (int j = 0; j < 7; j++) A[i * 7 + j] = KE[(i + 1) * 8 + (j + 1)];
      b[i] = feMu[(i + 1) * 3 + c];
    }
    lu_solve(7, A, b);
    disp[0 * 3 + c] = 0.0;
    for (int i = 0; i < 7; i++) disp[(i + 1) * 3 + c] = b[i];
  }
}

// ---------------------------------------------------------------------------------------
// Multigrid hierarchy in FP64: level 0 is matrix-free from k_e and KE
// (homogenization/grid.cu:318-471 operator action), coarse levels hold Galerkin 27-point
// stencils P^T A P with trilinear P (homogenization/grid_ex.cu:16-227).
// ---------------------------------------------------------------------------------------
struct Level {
  Dims d;
  std::vector<double> st;  // 27 * nv, st[o * nv + v], o = (ox+1) + 3(oy+1) + 9(oz+1)
  std::vector<double> u, f, r;
};

struct Hierarchy {
  std::vector<Level> lv;
  const double* ke = nullptr;  // fine element conductivity incl. the 1e-9 floor
  double KE[64];
  // coarsest dense factor
  int nc = 0;
  std::vector<double> L;  // Cholesky factor of A_c + alpha/n 11^T
  int pre = 2, post = 2;

  // 27-point row of the operator at vertex v of level l.
  void stencil(int l, size_t v, double s[27]) const {
    const Level& L0 = lv[l];
    if (l > 0) {
      for (int o = 0; o < 27; o++) s[o] = L0.st[o * L0.d.nv() + v];
      return;
    }
    const Dims& d = L0.d;
    int x = int(v % d.n[0]), y = int((v / d.n[0]) % d.n[1]), z = int(v / (size_t(d.n[0]) * d.n[1]));
    for (int o = 0; o < 27; o++) s[o] = 0.0;
    // the 8 elements around v: element ei has its lower corner at v - 1 + (ei bits) and
    // holds v as local node 7 - ei (homogenization/homoCommon.cuh:287-355, grid.cu:407-425)
    for (int ei = 0; ei < 8; ei++) {
      int ex = x - 1 + (ei & 1), ey = y - 1 + ((ei >> 1) & 1), ez = z - 1 + (ei >> 2);
      double k = ke[d.id(ex, ey, ez)];
      int self = 7 - ei;
      for (int j = 0; j < 8; j++) {
        int o = ((ei & 1) + (j & 1)) + 3 * (((ei >> 1) & 1) + ((j >> 1) & 1)) + 9 * ((ei >> 2) + (j >> 2));
        s[o] += k * KE[self * 8 + j];
      }
    }
  }

  size_t nb(const Dims& d, size_t v, int o) const {
    int x = int(v % d.n[0]), y = int((v / d.n[0]) % d.n[1]), z = int(v / (size_t(d.n[0]) * d.n[1]));
    return d.id(x + o % 3 - 1, y + (o / 3) % 3 - 1, z + o / 9 - 1);
  }

  void apply(int l, const double* u, double* y) const {
    const Dims& d = lv[l].d;
    const long long nv = (long long)d.nv();
#pragma omp parallel for schedule(static)
    for (long long v = 0; v < nv; v++) {
      double s[27];
      stencil(l, size_t(v), s);
      double acc = 0.0;
      for (int o = 0; o < 27; o++) acc += s[o] * u[nb(d, size_t(v), o)];
      y[v] = acc;
    }
  }

  // 8-colour Gauss-Seidel, colour = x%2 + 2(y%2) + 4(z%2), omega = 1
  // (homogenization/grid.cu:318-471 fine, :707-809 coarse; the colour loop at grid.cu:957-982).
  void gs(int l, bool reverse) {
    Level& L0 = lv[l];
    const Dims& d = L0.d;
    for (int cc = 0; cc < 8; cc++) {
      int c = reverse ? 7 - cc : cc;
      int cx = c & 1, cy = (c >> 1) & 1, cz = c >> 2;
#pragma omp parallel for collapse(2) schedule(static)
      for (int z = cz; z < d.n[2]; z += 2)
        for (int y = cy; y < d.n[1]; y += 2)
          for (int x = cx; x < d.n[0]; x += 2) {
            size_t v = d.id(x, y, z);
            double s[27];
            stencil(l, v, s);
            double acc = L0.f[v];
            for (int o = 0; o < 27; o++)
              if (o != 13) acc -= s[o] * L0.u[nb(d, v, o)];
            L0.u[v] = acc / s[13];
          }
    }
  }

  void residual(int l) {
    Level& L0 = lv[l];
    apply(l, L0.u.data(), L0.r.data());
    const long long nv = (long long)L0.d.nv();
#pragma omp parallel for schedule(static)
    for (long long v = 0; v < nv; v++) L0.r[v] = L0.f[v] - L0.r[v];
  }

  // f_c(V) = sum_d w(d) r(2V + d), full weighting = P^T (homogenization/grid.cu:811-878)
  void restrict_to(int l) {
    const Level& F = lv[l];
    Level& C = lv[l + 1];
    const Dims& dc = C.d;
    const long long nvc = (long long)dc.nv();
#pragma omp parallel for schedule(static)
    for (long long V = 0; V < nvc; V++) {
      int X = int(V % dc.n[0]), Y = int((V / dc.n[0]) % dc.n[1]), Z = int(V / (size_t(dc.n[0]) * dc.n[1]));
      double acc = 0.0;
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            double w = (1.0 - 0.5 * std::abs(dx)) * (1.0 - 0.5 * std::abs(dy)) * (1.0 - 0.5 * std::abs(dz));
            acc += w * F.r[F.d.id(2 * X + dx, 2 * Y + dy, 2 * Z + dz)];
          }
      C.f[V] = acc;
    }
  }

  // u_f += P u_c, trilinear (homogenization/grid.cu:881-940)
  void prolong_add(int l) {
    Level& F = lv[l];
    const Level& C = lv[l + 1];
    const Dims& df = F.d;
    const long long nvf = (long long)df.nv();
#pragma omp parallel for schedule(static)
    for (long long v = 0; v < nvf; v++) {
      int x = int(v % df.n[0]), y = int((v / df.n[0]) % df.n[1]), z = int(v / (size_t(df.n[0]) * df.n[1]));
      int cx[2], cy[2], cz[2];
      double wx[2], wy[2], wz[2];
      int nx = (x & 1) ? 2 : 1, ny = (y & 1) ? 2 : 1, nz = (z & 1) ? 2 : 1;
      cx[0] = x >> 1; cx[1] = (x + 1) >> 1; wx[0] = wx[1] = (x & 1) ? 0.5 : 1.0;
      cy[0] = y >> 1; cy[1] = (y + 1) >> 1; wy[0] = wy[1] = (y & 1) ? 0.5 : 1.0;
      cz[0] = z >> 1; cz[1] = (z + 1) >> 1; wz[0] = wz[1] = (z & 1) ? 0.5 : 1.0;
      double acc = 0.0;
      for (int a = 0; a < nz; a++)
        for (int b = 0; b < ny; b++)
          for (int c = 0; c < nx; c++) acc += wx[c] * wy[b] * wz[a] * C.u[C.d.id(cx[c], cy[b], cz[a])];
      F.u[v] += acc;
    }
  }

  // Galerkin coarse stencil P^T A_l P for level l+1 (homogenization/grid_ex.cu:16-227).
  void galerkin(int l) {
    const Level& F = lv[l];
    Level& C = lv[l + 1];
    const Dims& dc = C.d;
    const size_t nvc = dc.nv();
    C.st.assign(27 * nvc, 0.0);
#pragma omp parallel for schedule(static)
    for (long long V = 0; V < (long long)nvc; V++) {
      int X = int(V % dc.n[0]), Y = int((V / dc.n[0]) % dc.n[1]), Z = int(V / (size_t(dc.n[0]) * dc.n[1]));
      double acc[27] = {};
      for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
          for (int dx = -1; dx <= 1; dx++) {
            double wv = (1.0 - 0.5 * std::abs(dx)) * (1.0 - 0.5 * std::abs(dy)) * (1.0 - 0.5 * std::abs(dz));
            double s[27];
            stencil(l, F.d.id(2 * X + dx, 2 * Y + dy, 2 * Z + dz), s);
            for (int o = 0; o < 27; o++) {
              if (s[o] == 0.0) continue;
              int t[3] = {dx + o % 3 - 1, dy + (o / 3) % 3 - 1, dz + o / 9 - 1};
              // per axis, the coarse offsets O with |t - 2 O| <= 1 and their weights
              int cnt[3], Os[3][2];
              double ws[3][2];
              for (int a = 0; a < 3; a++) {
                switch (t[a]) {
                  case -2: cnt[a] = 1; Os[a][0] = -1; ws[a][0] = 1.0; break;
                  case -1: cnt[a] = 2; Os[a][0] = -1; ws[a][0] = 0.5; Os[a][1] = 0; ws[a][1] = 0.5; break;
                  case 0: cnt[a] = 1; Os[a][0] = 0; ws[a][0] = 1.0; break;
                  case 1: cnt[a] = 2; Os[a][0] = 0; ws[a][0] = 0.5; Os[a][1] = 1; ws[a][1] = 0.5; break;
                  default: cnt[a] = 1; Os[a][0] = 1; ws[a][0] = 1.0; break;
                }
              }
              for (int iz = 0; iz < cnt[2]; iz++)
                for (int iy = 0; iy < cnt[1]; iy++)
                  for (int ix = 0; ix < cnt[0]; ix++) {
                    int O = (Os[0][ix] + 1) + 3 * (Os[1][iy] + 1) + 9 * (Os[2][iz] + 1);
                    acc[O] += wv * s[o] * ws[0][ix] * ws[1][iy] * ws[2][iz];
                  }
            }
          }
      for (int o = 0; o < 27; o++) C.st[o * nvc + V] = acc[o];
    }
  }

  // Coarsest level: dense Cholesky of A + (alpha/n) 1 1^T, which is SPD on the periodic
  // nullspace (replaces the host BiCGSTAB + nullspace projection, homogenization/grid.cpp:272-310).
  void factor_coarsest() {
    int l = int(lv.size()) - 1;
    const Dims& d = lv[l].d;
    nc = int(d.nv());
    std::vector<double> A(size_t(nc) * nc, 0.0);
    double diag = 0.0;
    for (int v = 0; v < nc; v++) {
      double s[27];
      stencil(l, size_t(v), s);
      for (int o = 0; o < 27; o++) A[size_t(v) * nc + nb(d, size_t(v), o)] += s[o];
      diag += s[13];
    }
    double alpha = diag / nc / nc;
    for (auto& a : A) a += alpha;
    L.assign(size_t(nc) * nc, 0.0);
    for (int j = 0; j < nc; j++) {
      double s = A[size_t(j) * nc + j];
      for (int k = 0; k < j; k++) s -= L[size_t(j) * nc + k] * L[size_t(j) * nc + k];
      double ljj = std::sqrt(std::max(s, 1e-300));
      L[size_t(j) * nc + j] = ljj;
      for (int i = j + 1; i < nc; i++) {
        double t = A[size_t(i) * nc + j];
        for (int k = 0; k < j; k++) t -= L[size_t(i) * nc + k] * L[size_t(j) * nc + k];
        L[size_t(i) * nc + j] = t / ljj;
      }
    }
  }

  void solve_coarsest() {
    Level& C = lv.back();
    std::vector<double> b(C.f.begin(), C.f.end());
    double mean = 0.0;
    for (double x : b) mean += x;
    mean /= nc;
    for (double& x : b) x -= mean;
    for (int i = 0; i < nc; i++) {
      double s = b[i];
      for (int k = 0; k < i; k++) s -= L[size_t(i) * nc + k] * b[k];
      b[i] = s / L[size_t(i) * nc + i];
    }
    for (int i = nc - 1; i >= 0; i--) {
      double s = b[i];
      for (int k = i + 1; k < nc; k++) s -= L[size_t(k) * nc + i] * b[k];
      b[i] = s / L[size_t(i) * nc + i];
    }
    for (int i = 0; i < nc; i++) C.u[i] = b[i];
  }

  // V-cycle with zero initial guess on level l: pre sweeps forward colours, post sweeps
  // reverse colours so that the cycle is a symmetric preconditioner (homogenization/MG.cpp:46-71).
  void vcycle(int l) {
    Level& F = lv[l];
    if (l == int(lv.size()) - 1) {
      solve_coarsest();
      return;
    }
    std::fill(F.u.begin(), F.u.end(), 0.0);
    for (int i = 0; i < pre; i++) gs(l, false);
    residual(l);
    restrict_to(l);
    vcycle(l + 1);
    prolong_add(l);
    for (int i = 0; i < post; i++) gs(l, true);
  }

  void build(const int n[3], const double* k, const double KEin[64], int coarsest_max_dof) {
    std::memcpy(KE, KEin, sizeof(KE));
    ke = k;
    lv.clear();
    Dims d{{n[0], n[1], n[2]}};
    while (true) {
      Level L0;
      L0.d = d;
      L0.u.assign(d.nv(), 0.0);
      L0.f.assign(d.nv(), 0.0);
      L0.r.assign(d.nv(), 0.0);
      lv.push_back(std::move(L0));
      bool can = d.n[0] % 2 == 0 && d.n[1] % 2 == 0 && d.n[2] % 2 == 0 && d.n[0] >= 8 && d.n[1] >= 8 &&
                 d.n[2] >= 8 && d.nv() > size_t(coarsest_max_dof);
      if (!can) break;
      d = Dims{{d.n[0] / 2, d.n[1] / 2, d.n[2] / 2}};
    }
    for (int l = 0; l + 1 < int(lv.size()); l++) galerkin(l);
    factor_coarsest();
  }
};

double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0.0;
  const long long n = (long long)a.size();
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long long i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}

void remove_mean(std::vector<double>& a) {
  double s = 0.0;
  const long long n = (long long)a.size();
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (long long i = 0; i < n; i++) s += a[i];
  s /= double(n);
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < n; i++) a[i] -= s;
}

// Preconditioned CG on the periodic (singular, consistent) system; the preconditioner is
// one symmetric V-cycle (precond = 1) or Jacobi (precond = 0). Iterates stay mean-free.
// The stopping rule is ||f - A x||_2 <= tol ||f||_2 (homogenization/MG.cpp:80-142).
int pcg(Hierarchy& H, const std::vector<double>& f, std::vector<double>& x, double tol, int max_iter, int precond,
        double* relres) {
  const size_t n = f.size();
  Level& L0 = H.lv[0];
  std::vector<double> r(n), z(n), p(n), q(n), diag;
  if (precond == 0) {
    diag.resize(n);
    for (size_t v = 0; v < n; v++) {
      double s[27];
      H.stencil(0, v, s);
      diag[v] = s[13];
    }
  }
  remove_mean(x);
  H.apply(0, x.data(), q.data());
  for (size_t i = 0; i < n; i++) r[i] = f[i] - q[i];
  // relative residual with the reference's absolute floor, homogenization/MG.cpp:391
  double fn = std::sqrt(dot(f, f)) + 1e-10;
  auto precondition = [&]() {
    if (precond == 0) {
      for (size_t i = 0; i < n; i++) z[i] = r[i] / diag[i];
    } else {
      std::copy(r.begin(), r.end(), L0.f.begin());
      H.vcycle(0);
      std::copy(L0.u.begin(), L0.u.end(), z.begin());
    }
    remove_mean(z);
  };
  double rn = std::sqrt(dot(r, r)) / fn;
  int it = 0;
  if (rn <= tol) {
    *relres = rn;
    return 0;
  }
  precondition();
  p = z;
  double rho = dot(r, z);
  for (it = 1; it <= max_iter; it++) {
    H.apply(0, p.data(), q.data());
    double alpha = rho / dot(p, q);
    for (size_t i = 0; i < n; i++) {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    rn = std::sqrt(dot(r, r)) / fn;
    if (rn <= tol) break;
    precondition();
    double rho2 = dot(r, z);
    double beta = rho2 / rho;
    rho = rho2;
    for (size_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
  }
  *relres = rn;
  return it;
}

// Element energies E_ij(e) = (chi0_i - chi_i)^T KE (chi0_j - chi_j), unique pairs in the
// order 00, 01, 02, 11, 12, 22 (homogenization/homogenization.cu:13-153, 255-412).
void element_energy(const Dims& d, const double KE[64], const double disp[24], const double* chi, size_t e,
                    double E[6]) {
  int x = int(e % d.n[0]), y = int((e / d.n[0]) % d.n[1]), z = int(e / (size_t(d.n[0]) * d.n[1]));
  double u[3][8];
  for (int j = 0; j < 8; j++) {
    size_t v = d.id(x + (j & 1), y + ((j >> 1) & 1), z + (j >> 2));
    for (int c = 0; c < 3; c++) u[c][j] = disp[j * 3 + c] - chi[c * d.nv() + v];
  }
  double Ku[3][8];
  for (int c = 0; c < 3; c++)
    for (int i = 0; i < 8; i++) {
      double s = 0.0;
      for (int j = 0; j < 8; j++) s += KE[i * 8 + j] * u[c][j];
      Ku[c][i] = s;
    }
  int cnt = 0;
  for (int a = 0; a < 3; a++)
    for (int b = a; b < 3; b++) {
      double s = 0.0;
      for (int i = 0; i < 8; i++) s += u[a][i] * Ku[b][i];
      E[cnt++] = s;
    }
}

// Radial weight functions and kernel enumeration (AutoDiff/TensorExpression.h:993-1093).
double radial_weight(int wtype, double r, int ox, int oy, int oz) {
  double q2 = double(ox * ox + oy * oy + oz * oz) / (r * r);
  double q = std::sqrt(q2);
  if (q2 >= 1.0) return 0.0;
  if (wtype == 0) return 1.0 - 6.0 * q2 + 8.0 * q2 * q - 3.0 * q2 * q2;  // Spline4
  return 1.0 - q;                                                      // Linear
}

}  // namespace

extern "C" {

// KE (8x8), feMu (8x3) and the element macro field disp (8x3) for a cell of reso voxels per
// axis, element half-length 1/(2 reso) (homogenization/homogenization.cpp:211).
void ora_template_matrix(int reso, double* KE, double* feMu, double* disp) {
  template_matrix(1.0 / reso / 2.0, KE, feMu, disp);
}

int ora_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void ora_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// y = A x with the fine-level operator for conductivity k (k already includes the 1e-9 floor).
void ora_apply(const int* n, const double* k_solver, const double* x, double* y) {
  Hierarchy H;
  double KE[64], fe[24], dp[24];
  template_matrix(1.0 / n[0] / 2.0, KE, fe, dp);
  std::memcpy(H.KE, KE, sizeof(KE));
  H.ke = k_solver;
  Level L0;
  L0.d = Dims{{n[0], n[1], n[2]}};
  H.lv.push_back(L0);
  H.apply(0, x, y);
}

// Load-case right-hand sides f_c(v) = sum_{e ni v} k_e feMu[local(v)][c]
// (homogenization/grid.cu:1282-1327); f is 3 * nv, case-major.
void ora_rhs(const int* n, const double* k_solver, double* f) {
  double KE[64], fe[24], dp[24];
  template_matrix(1.0 / n[0] / 2.0, KE, fe, dp);
  Dims d{{n[0], n[1], n[2]}};
  const long long nv = (long long)d.nv();
#pragma omp parallel for schedule(static)
  for (long long v = 0; v < nv; v++) {
    int x = int(v % d.n[0]), y = int((v / d.n[0]) % d.n[1]), z = int(v / (size_t(d.n[0]) * d.n[1]));
    double acc[3] = {0, 0, 0};
    for (int ei = 0; ei < 8; ei++) {
      double k = k_solver[d.id(x - 1 + (ei & 1), y - 1 + ((ei >> 1) & 1), z - 1 + (ei >> 2))];
      for (int c = 0; c < 3; c++) acc[c] += k * fe[(7 - ei) * 3 + c];
    }
    for (int c = 0; c < 3; c++) f[c * nv + v] = acc[c];
  }
}

// Full homogenization of a cell: k_in is the conductivity handed to update(); the solver
// uses 1e-9 + k_in^power_penal. Solves the 3 load cases to ||r||/||f|| <= tol, returns K^H
// (reference axis convention, volume 1) and optionally chi (3 * nv) and the element
// energies (6 * ne, pairs 00 01 02 11 12 22). precond: 1 = MG V(2,2), 0 = Jacobi.
// Returns the largest PCG iteration count, or -1 if a case did not converge.
int ora_homogenize_cases(const int* n, const double* k_in, double power_penal, double tol, int max_iter,
                         int precond, int coarsest_max_dof, int case_mask, double* C, double* chi_out,
                         double* energy_out, double* relres_out);

int ora_homogenize(const int* n, const double* k_in, double power_penal, double tol, int max_iter, int precond,
                   int coarsest_max_dof, double* C, double* chi_out, double* energy_out, double* relres_out) {
  return ora_homogenize_cases(n, k_in, power_penal, tol, max_iter, precond, coarsest_max_dof, 7, C, chi_out,
                              energy_out, relres_out);
}

// As ora_homogenize, solving only the load cases whose bit is set in case_mask (the others
// keep chi = 0); used to time bounded samples of a solve.
int ora_homogenize_cases(const int* n, const double* k_in, double power_penal, double tol, int max_iter,
                         int precond, int coarsest_max_dof, int case_mask, double* C, double* chi_out,
                         double* energy_out, double* relres_out) {
  Dims d{{n[0], n[1], n[2]}};
  const size_t nv = d.nv();
  std::vector<double> ks(nv);
  for (size_t e = 0; e < nv; e++) ks[e] = kRhoPenalMin + std::pow(k_in[e], power_penal);
  double KE[64], fe[24], dp[24];
  template_matrix(1.0 / n[0] / 2.0, KE, fe, dp);
  Hierarchy H;
  H.build(n, ks.data(), KE, coarsest_max_dof > 0 ? coarsest_max_dof : 64);
  std::vector<double> f(3 * nv);
  ora_rhs(n, ks.data(), f.data());
  std::vector<double> chi(3 * nv, 0.0);
  int worst = 0;
  for (int c = 0; c < 3; c++) {
    if (!(case_mask & (1 << c))) {
      if (relres_out) relres_out[c] = 0.0;
      continue;
    }
    std::vector<double> fc(f.begin() + c * nv, f.begin() + (c + 1) * nv);
    remove_mean(fc);
    std::vector<double> x(nv, 0.0);
    double rr = 0.0;
    int it = pcg(H, fc, x, tol, max_iter, precond, &rr);
    if (relres_out) relres_out[c] = rr;
    if (rr > tol) worst = -1;
    if (worst >= 0) worst = std::max(worst, it);
    std::copy(x.begin(), x.end(), chi.begin() + c * nv);
  }
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const long long ne = (long long)nv;
#pragma omp parallel
  {
    double loc[6] = {0, 0, 0, 0, 0, 0};
#pragma omp for schedule(static)
    for (long long e = 0; e < ne; e++) {
      double E[6];
      element_energy(d, KE, dp, chi.data(), size_t(e), E);
      if (energy_out)
        for (int q = 0; q < 6; q++) energy_out[q * nv + e] = E[q];
      for (int q = 0; q < 6; q++) loc[q] += ks[e] * E[q];
    }
#pragma omp critical
    for (int q = 0; q < 6; q++) acc[q] += loc[q];
  }
  // vol = 1 (homogenization/homogenization.cu:189-236)
  int cnt = 0;
  for (int a = 0; a < 3; a++)
    for (int b = a; b < 3; b++) {
      C[a * 3 + b] = acc[cnt];
      C[b * 3 + a] = acc[cnt];
      cnt++;
    }
  if (chi_out) std::copy(chi.begin(), chi.end(), chi_out);
  return worst;
}

// As ora_homogenize for the 3 load cases, with chi_inout (3 * nv) as the initial guess of every
// case and the solutions written back to it: the warm-started solve of an optimisation loop
// (homogenization/homogenization.cu:182-188 keeps each case's last solution as its next initial
// guess). One hierarchy build per call. iters_out (3, optional) gets each case's PCG iterations.
int ora_homogenize_warm(const int* n, const double* k_in, double power_penal, double tol, int max_iter, int precond,
                        int coarsest_max_dof, double* chi_inout, double* C, double* energy_out, double* relres_out,
                        int* iters_out) {
  Dims d{{n[0], n[1], n[2]}};
  const size_t nv = d.nv();
  std::vector<double> ks(nv);
  for (size_t e = 0; e < nv; e++) ks[e] = kRhoPenalMin + std::pow(k_in[e], power_penal);
  double KE[64], fe[24], dp[24];
  template_matrix(1.0 / n[0] / 2.0, KE, fe, dp);
  Hierarchy H;
  H.build(n, ks.data(), KE, coarsest_max_dof > 0 ? coarsest_max_dof : 64);
  std::vector<double> f(3 * nv);
  ora_rhs(n, ks.data(), f.data());
  int worst = 0;
  for (int c = 0; c < 3; c++) {
    std::vector<double> fc(f.begin() + c * nv, f.begin() + (c + 1) * nv);
    remove_mean(fc);
    std::vector<double> x(chi_inout + c * nv, chi_inout + (c + 1) * nv);
    double rr = 0.0;
    int it = pcg(H, fc, x, tol, max_iter, precond, &rr);
    if (relres_out) relres_out[c] = rr;
    if (iters_out) iters_out[c] = it;
    if (rr > tol) worst = -1;
    if (worst >= 0) worst = std::max(worst, it);
    std::copy(x.begin(), x.end(), chi_inout + c * nv);
  }
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const long long ne = (long long)nv;
#pragma omp parallel
  {
    double loc[6] = {0, 0, 0, 0, 0, 0};
#pragma omp for schedule(static)
    for (long long e = 0; e < ne; e++) {
      double E[6];
      element_energy(d, KE, dp, chi_inout, size_t(e), E);
      if (energy_out)
        for (int q = 0; q < 6; q++) energy_out[q * nv + e] = E[q];
      for (int q = 0; q < 6; q++) loc[q] += ks[e] * E[q];
    }
#pragma omp critical
    for (int q = 0; q < 6; q++) acc[q] += loc[q];
  }
  int cnt = 0;
  for (int a = 0; a < 3; a++)
    for (int b = a; b < 3; b++) {
      C[a * 3 + b] = acc[cnt];
      C[b * 3 + a] = acc[cnt];
      cnt++;
    }
  return worst;
}

// Element energies for a given chi (3 * nv), pairs 00 01 02 11 12 22.
void ora_element_energy(const int* n, const double* chi, double* energy_out) {
  Dims d{{n[0], n[1], n[2]}};
  double KE[64], fe[24], dp[24];
  template_matrix(1.0 / n[0] / 2.0, KE, fe, dp);
  const long long ne = (long long)d.nv();
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < ne; e++) {
    double E[6];
    element_energy(d, KE, dp, chi, size_t(e), E);
    for (int q = 0; q < 6; q++) energy_out[q * ne + e] = E[q];
  }
}

// s_e = p k_e^(p-1) sum_{i<=j} E_ij(e) (dC_ij + [i != j] dC_ji) / vol
// (homogenization/homogenization.cu:255-412, 415-479).
void ora_sensitivity(const int* n, const double* energy, const double* k_in, double power_penal, const double* dC,
                     double* sens) {
  const long long ne = (long long)n[0] * n[1] * n[2];
#pragma omp parallel for schedule(static)
  for (long long e = 0; e < ne; e++) {
    double pr = power_penal * std::pow(k_in[e], power_penal - 1.0);
    double s = 0.0;
    int cnt = 0;
    for (int a = 0; a < 3; a++)
      for (int b = a; b < 3; b++) {
        double w = dC[a * 3 + b] + (a != b ? dC[b * 3 + a] : 0.0);
        s += energy[cnt * ne + e] * w;
        cnt++;
      }
    sens[e] = s * pr;
  }
}

// Density filter forward: dst = sum w src / sum_valid w, wsum_out = sum_valid w; wtype 0 =
// Spline4, 1 = Linear; halfwidth = int(r + 0.5); zero padding unless periodic
// (AutoDiff/TensorExpression.cuh:304-350, TensorExpression.h:993-1093).
void ora_conv_forward(const int* n, const double* src, double* dst, double* wsum_out, int wtype, double radius,
                      int periodic) {
  int hw = int(radius + 0.5);
  double wtot = 0.0;
  for (int oz = -hw; oz <= hw; oz++)
    for (int oy = -hw; oy <= hw; oy++)
      for (int ox = -hw; ox <= hw; ox++) wtot += radial_weight(wtype, radius, ox, oy, oz);
  Dims d{{n[0], n[1], n[2]}};
  const long long nv = (long long)d.nv();
#pragma omp parallel for schedule(static)
  for (long long v = 0; v < nv; v++) {
    int x = int(v % d.n[0]), y = int((v / d.n[0]) % d.n[1]), z = int(v / (size_t(d.n[0]) * d.n[1]));
    double sum = 0.0, ws = 0.0;
    for (int oz = -hw; oz <= hw; oz++)
      for (int oy = -hw; oy <= hw; oy++)
        for (int ox = -hw; ox <= hw; ox++) {
          double w = radial_weight(wtype, radius, ox, oy, oz) / wtot;
          int px = x + ox, py = y + oy, pz = z + oz;
          bool in = px >= 0 && px < d.n[0] && py >= 0 && py < d.n[1] && pz >= 0 && pz < d.n[2];
          if (in || periodic) {
            sum += w * src[d.id(px, py, pz)];
            ws += w;
          }
        }
    dst[v] = sum / ws;
    if (wsum_out) wsum_out[v] = ws;
  }
}

// Adjoint of ora_conv_forward: g_src(i) = sum_off w(off) g_dst(i - off) / ws(i - off)
// (AutoDiff/TensorExpression.cuh:353-385).
void ora_conv_backward(const int* n, const double* g_dst, const double* wsum, double* g_src, int wtype,
                       double radius, int periodic) {
  int hw = int(radius + 0.5);
  double wtot = 0.0;
  for (int oz = -hw; oz <= hw; oz++)
    for (int oy = -hw; oy <= hw; oy++)
      for (int ox = -hw; ox <= hw; ox++) wtot += radial_weight(wtype, radius, ox, oy, oz);
  Dims d{{n[0], n[1], n[2]}};
  const long long nv = (long long)d.nv();
#pragma omp parallel for schedule(static)
  for (long long v = 0; v < nv; v++) {
    int x = int(v % d.n[0]), y = int((v / d.n[0]) % d.n[1]), z = int(v / (size_t(d.n[0]) * d.n[1]));
    double sum = 0.0;
    for (int oz = -hw; oz <= hw; oz++)
      for (int oy = -hw; oy <= hw; oy++)
        for (int ox = -hw; ox <= hw; ox++) {
          double w = radial_weight(wtype, radius, ox, oy, oz) / wtot;
          int px = x - ox, py = y - oy, pz = z - oz;
          bool in = px >= 0 && px < d.n[0] && py >= 0 && py < d.n[1] && pz >= 0 && pz < d.n[2];
          if (in || periodic) {
            size_t q = d.id(px, py, pz);
            sum += w * g_dst[q] / wsum[q];
          }
        }
    g_src[v] = sum;
  }
}

// OC sensitivity filter, periodic Linear weights of radius r (optimization/OCOptimizer.cu:76-104, 134-152).
void ora_oc_filter_sens(const int* n, double* sens, const double* rho, double radius) {
  int hw = int(radius + 0.5);
  double wtot = 0.0;
  for (int oz = -hw; oz <= hw; oz++)
    for (int oy = -hw; oy <= hw; oy++)
      for (int ox = -hw; ox <= hw; ox++) wtot += radial_weight(1, radius, ox, oy, oz);
  Dims d{{n[0], n[1], n[2]}};
  const long long nv = (long long)d.nv();
  std::vector<double> out(nv);
#pragma omp parallel for schedule(static)
  for (long long v = 0; v < nv; v++) {
    int x = int(v % d.n[0]), y = int((v / d.n[0]) % d.n[1]), z = int(v / (size_t(d.n[0]) * d.n[1]));
    double sum = 0.0, ws = 0.0;
    for (int oz = -hw; oz <= hw; oz++)
      for (int oy = -hw; oy <= hw; oy++)
        for (int ox = -hw; ox <= hw; ox++) {
          double w = radial_weight(1, radius, ox, oy, oz) / wtot;
          size_t q = d.id(x + ox, y + oy, z + oz);
          sum += sens[q] * rho[q] * w;
          ws += w;
        }
    out[v] = sum / (ws * rho[v]);
  }
  std::copy(out.begin(), out.end(), sens);
}

// OC update: bisection on the multiplier g in [0, max|sens|], at most 20 steps, stop when the
// volume is within 1e-4 of the target (optimization/OCOptimizer.cu:12-67). Returns steps used.
int ora_oc_update(long long ne, const double* sens, double* rho, double volratio, double min_rho, double step_limit,
                  double damp) {
  double maxs = 0.0;
  for (long long i = 0; i < ne; i++) maxs = std::max(maxs, std::fabs(sens[i]));
  double mins = 0.0;
  std::vector<double> nr(ne);
  int it;
  for (it = 0; it < 20; it++) {
    double g = (maxs + mins) / 2.0;
    double vol = 0.0;
#pragma omp parallel for reduction(+ : vol) schedule(static)
    for (long long i = 0; i < ne; i++) {
      double r = rho[i];
      double B = -sens[i] / g;
      if (B < 0) B = 0.01;
      double x = std::pow(B, damp) * r;
      if (x - r < -step_limit) x = r - step_limit;
      if (x - r > step_limit) x = r + step_limit;
      if (x < min_rho) x = min_rho;
      if (x > 1) x = 1;
      nr[i] = x;
      vol += x;
    }
    vol /= double(ne);
    if (vol < volratio - 1e-4)
      maxs = g;
    else if (vol > volratio + 1e-4)
      mins = g;
    else {
      it++;
      break;
    }
  }
  std::copy(nr.begin(), nr.end(), rho);
  return it;
}

// One MMA step (Svanberg's method of moving asymptotes), FP64, m constraints, n variables;
// dgdx is m x n row-major. Updates xvar, xold1, xold2, low, upp in place
// (optimization/mmaOpt.cu:834-1019 mmasub_ker, 429-830 subsolv_g, mmaOpt.cpp:48-73).
void ora_mmasub(int m, long long n, int itn, double* xvar, const double* xmin, const double* xmax, double* xold1,
                double* xold2, const double* df0dx, const double* gval, const double* dgdx, double* low,
                double* upp, double a0, const double* a, const double* c, const double* d, double move) {
  const double epsimin = 1e-7, raa0 = 1e-5, albefa = 0.1, asyinit = 0.5, asyincr = 1.2, asydecr = 0.7;
  typedef std::vector<double> V;
  V x(xvar, xvar + n);
  if (itn <= 2) {
    for (long long j = 0; j < n; j++) {
      low[j] = x[j] - asyinit * (xmax[j] - xmin[j]);
      upp[j] = x[j] + asyinit * (xmax[j] - xmin[j]);
    }
  } else {
    for (long long j = 0; j < n; j++) {
      double zzz = (x[j] - xold1[j]) * (xold1[j] - xold2[j]);
      double f = 1.0;
      if (zzz > 0) f = asyincr;
      if (zzz < 0) f = asydecr;
      double lo = x[j] - f * (xold1[j] - low[j]);
      double up = x[j] + f * (upp[j] - xold1[j]);
      double dx = xmax[j] - xmin[j];
      lo = std::max(lo, x[j] - 10 * dx);
      lo = std::min(lo, x[j] - 0.01 * dx);
      up = std::min(up, x[j] + 10 * dx);
      up = std::max(up, x[j] + 0.01 * dx);
      low[j] = lo;
      upp[j] = up;
    }
  }
  V alfa(n), beta(n), p0(n), q0(n), P(size_t(m) * n), Q(size_t(m) * n), b(m, 0.0);
  for (long long j = 0; j < n; j++) {
    double dxr = xmax[j] - xmin[j];
    alfa[j] = std::max(std::max(low[j] + albefa * (x[j] - low[j]), x[j] - move * dxr), xmin[j]);
    beta[j] = std::min(std::min(upp[j] - albefa * (upp[j] - x[j]), x[j] + move * dxr), xmax[j]);
    double xmamiinv = 1.0 / std::max(dxr, 1e-5);
    double ux1 = upp[j] - x[j], xl1 = x[j] - low[j];
    double ux2 = ux1 * ux1, xl2 = xl1 * xl1;
    double dp = std::max(df0dx[j], 0.0), dm = std::max(-df0dx[j], 0.0);
    double pq0 = 1e-3 * (dp + dm) + raa0 * xmamiinv;
    p0[j] = (dp + pq0) * ux2;
    q0[j] = (dm + pq0) * xl2;
    for (int i = 0; i < m; i++) {
      double g = dgdx[size_t(i) * n + j];
      double pp = std::max(g, 0.0), qq = std::max(-g, 0.0);
      double pq = 1e-3 * (pp + qq) + raa0 * xmamiinv;
      P[size_t(i) * n + j] = (pp + pq) * ux2;
      Q[size_t(i) * n + j] = (qq + pq) * xl2;
      b[i] += P[size_t(i) * n + j] / ux1 + Q[size_t(i) * n + j] / xl1;
    }
  }
  for (int i = 0; i < m; i++) b[i] -= gval[i];

  // ---- subsolv (optimization/mmaOpt.cu:429-830) ----
  V xs(n), xsi(n), eta(n);
  for (long long j = 0; j < n; j++) {
    xs[j] = 0.5 * (alfa[j] + beta[j]);
    xsi[j] = std::max(1.0 / (xs[j] - alfa[j]), 1.0);
    eta[j] = std::max(1.0 / (beta[j] - xs[j]), 1.0);
  }
  V y(m, 1.0), lam(m, 1.0), mu(m), s(m, 1.0);
  for (int i = 0; i < m; i++) mu[i] = std::max(0.5 * c[i], 1.0);
  double z = 1.0, zet = 1.0, epsi = 1.0;
  V plam(n), qlam(n), gvec(m);
  auto pq_update = [&](const V& xx, const V& ll) {
    for (int i = 0; i < m; i++) gvec[i] = 0.0;
    for (long long j = 0; j < n; j++) {
      double ps = p0[j], qs = q0[j];
      double uxi = 1.0 / (upp[j] - xx[j]), xli = 1.0 / (xx[j] - low[j]);
      for (int i = 0; i < m; i++) {
        ps += P[size_t(i) * n + j] * ll[i];
        qs += Q[size_t(i) * n + j] * ll[i];
        gvec[i] += P[size_t(i) * n + j] * uxi + Q[size_t(i) * n + j] * xli;
      }
      plam[j] = ps;
      qlam[j] = qs;
    }
  };
  auto residual = [&](const V& xx, const V& yy, double zz, const V& ll, const V& xs_, const V& et, const V& mm,
                      double ze, const V& ss, double* nrm, double* mx) {
    pq_update(xx, ll);
    double n2 = 0.0, am = 0.0;
    auto acc = [&](double r) {
      n2 += r * r;
      am = std::max(am, std::fabs(r));
    };
    for (long long j = 0; j < n; j++) {
      double ux1 = upp[j] - xx[j], xl1 = xx[j] - low[j];
      double dpsidx = plam[j] / (ux1 * ux1) - qlam[j] / (xl1 * xl1);
      acc(dpsidx - xs_[j] + et[j]);
    }
    for (int i = 0; i < m; i++) acc(c[i] + d[i] * yy[i] - mm[i] - ll[i]);
    double ad = 0.0;
    for (int i = 0; i < m; i++) ad += a[i] * ll[i];
    acc(a0 - ze - ad);
    for (int i = 0; i < m; i++) acc(gvec[i] - a[i] * zz - yy[i] + ss[i] - b[i]);
    for (long long j = 0; j < n; j++) acc(xs_[j] * (xx[j] - alfa[j]) - epsi);
    for (long long j = 0; j < n; j++) acc(et[j] * (beta[j] - xx[j]) - epsi);
    for (int i = 0; i < m; i++) acc(mm[i] * yy[i] - epsi);
    acc(ze * zz - epsi);
    for (int i = 0; i < m; i++) acc(ll[i] * ss[i] - epsi);
    *nrm = std::sqrt(n2);
    *mx = am;
  };
  V delx(n), diagx(n), dx(n), dxsi(n), deta(n), GG(size_t(m) * n);
  V dely(m), dellam(m), diagy(m), dy(m), dlam(m), dmu(m), ds(m);
  while (epsi > epsimin) {
    double residunorm, residumax;
    residual(xs, y, z, lam, xsi, eta, mu, zet, s, &residunorm, &residumax);
    int ittt = 0;
    while (residumax > 0.9 * epsi && ittt < 200) {
      ittt++;
      pq_update(xs, lam);
      for (long long j = 0; j < n; j++) {
        double ux1 = upp[j] - xs[j], xl1 = xs[j] - low[j];
        double ux2 = ux1 * ux1, xl2 = xl1 * xl1, ux3 = ux1 * ux2, xl3 = xl1 * xl2;
        for (int i = 0; i < m; i++) GG[size_t(i) * n + j] = P[size_t(i) * n + j] / ux2 - Q[size_t(i) * n + j] / xl2;
        double dpsidx = plam[j] / ux2 - qlam[j] / xl2;
        delx[j] = dpsidx - epsi / (xs[j] - alfa[j]) + epsi / (beta[j] - xs[j]);
        diagx[j] = 2 * (plam[j] / ux3 + qlam[j] / xl3) + xsi[j] / (xs[j] - alfa[j]) + eta[j] / (beta[j] - xs[j]);
      }
      double adl = 0.0;
      for (int i = 0; i < m; i++) adl += a[i] * lam[i];
      double delz = a0 - adl - epsi / z;
      for (int i = 0; i < m; i++) {
        dely[i] = c[i] + d[i] * y[i] - lam[i] - epsi / y[i];
        dellam[i] = gvec[i] - a[i] * z - y[i] - b[i] + epsi / lam[i];
        diagy[i] = d[i] + mu[i] / y[i];
      }
      // (m+1) x (m+1) KKT system, solved densely (replaces Eigen ColPivHouseholderQR)
      std::vector<double> AA(size_t(m + 1) * (m + 1), 0.0);
      std::vector<double> bb(m + 1);
      for (int i = 0; i < m; i++) {
        double gx = 0.0;
        for (long long j = 0; j < n; j++) gx += GG[size_t(i) * n + j] * delx[j] / diagx[j];
        bb[i] = dellam[i] + dely[i] / diagy[i] - gx;
        for (int k = 0; k < m; k++) {
          double sacc = 0.0;
          for (long long j = 0; j < n; j++) sacc += GG[size_t(i) * n + j] * GG[size_t(k) * n + j] / diagx[j];
          AA[size_t(i) * (m + 1) + k] = sacc;
        }
        AA[size_t(i) * (m + 1) + i] += s[i] / lam[i] + 1.0 / diagy[i];
        AA[size_t(i) * (m + 1) + m] = a[i];
        AA[size_t(m) * (m + 1) + i] = a[i];
      }
      AA[size_t(m) * (m + 1) + m] = -zet / z;
      bb[m] = delz;
      lu_solve(m + 1, AA, bb.data());
      for (int i = 0; i < m; i++) dlam[i] = bb[i];
      double dz = bb[m];
      for (long long j = 0; j < n; j++) {
        double gl = 0.0;
        for (int i = 0; i < m; i++) gl += GG[size_t(i) * n + j] * dlam[i];
        dx[j] = -delx[j] / diagx[j] - gl / diagx[j];
        dxsi[j] = -xsi[j] + epsi / (xs[j] - alfa[j]) - (xsi[j] * dx[j]) / (xs[j] - alfa[j]);
        deta[j] = -eta[j] + epsi / (beta[j] - xs[j]) + (eta[j] * dx[j]) / (beta[j] - xs[j]);
      }
      for (int i = 0; i < m; i++) {
        dy[i] = -dely[i] / diagy[i] + dlam[i] / diagy[i];
        dmu[i] = -mu[i] + epsi / y[i] - (mu[i] * dy[i]) / y[i];
        ds[i] = -s[i] + epsi / lam[i] - (s[i] * dlam[i]) / lam[i];
      }
      double dzet = -zet + epsi / z - zet * dz / z;
      // step length from the positivity constraints
      double stm = -1e300;
      auto upd = [&](double v) { stm = std::max(stm, v); };
      for (int i = 0; i < m; i++) upd(-1.01 * dy[i] / y[i]);
      upd(-1.01 * dz / z);
      for (int i = 0; i < m; i++) upd(-1.01 * dlam[i] / lam[i]);
      for (long long j = 0; j < n; j++) upd(-1.01 * dxsi[j] / xsi[j]);
      for (long long j = 0; j < n; j++) upd(-1.01 * deta[j] / eta[j]);
      for (int i = 0; i < m; i++) upd(-1.01 * dmu[i] / mu[i]);
      upd(-1.01 * dzet / zet);
      for (int i = 0; i < m; i++) upd(-1.01 * ds[i] / s[i]);
      double stmalfa = -1e300, stmbeta = -1e300;
      for (long long j = 0; j < n; j++) {
        stmalfa = std::max(stmalfa, -1.01 * dx[j] / (xs[j] - alfa[j]));
        stmbeta = std::max(stmbeta, 1.01 * dx[j] / (beta[j] - xs[j]));
      }
      double stminv = std::max(std::max(std::max(stmalfa, stmbeta), stm), 1.0);
      double steg = 1.0 / stminv;
      V xold = xs, yold = y, lamold = lam, xsiold = xsi, etaold = eta, muold = mu, sold = s;
      double zold = z, zetold = zet;
      int itto = 0;
      double resinew = 2 * residunorm, resimax = residumax;
      while (resinew > residunorm && itto < 50) {
        itto++;
        for (long long j = 0; j < n; j++) {
          xs[j] = xold[j] + steg * dx[j];
          xsi[j] = xsiold[j] + steg * dxsi[j];
          eta[j] = etaold[j] + steg * deta[j];
        }
        for (int i = 0; i < m; i++) {
          y[i] = yold[i] + steg * dy[i];
          lam[i] = lamold[i] + steg * dlam[i];
          mu[i] = muold[i] + steg * dmu[i];
          s[i] = sold[i] + steg * ds[i];
        }
        z = zold + steg * dz;
        zet = zetold + steg * dzet;
        residual(xs, y, z, lam, xsi, eta, mu, zet, s, &resinew, &resimax);
        steg /= 2;
      }
      residunorm = resinew;
      residumax = resimax;
    }
    epsi *= 0.1;
  }
  for (long long j = 0; j < n; j++) {
    xold2[j] = xold1[j];
    xold1[j] = xvar[j];
    xvar[j] = xs[j];
  }
}

}  // extern "C"
