// fe.cpp -- host-side FE and homogenisation helpers (FP64).
#include "fe.h"

#include "ddmath.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace dtc {
namespace {

const double kPi = std::acos(-1.0);
const double kPiDiv180 = kPi / 180.0;
const double kSqrt2 = std::sqrt(2.0);

// local node positions in [-1,1]^3
const signed char kCorner8[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                                    {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
const signed char kRing20[20][3] = {{-1, -1, -1}, {0, -1, -1}, {1, -1, -1}, {1, 0, -1}, {1, 1, -1},
                                    {0, 1, -1},   {-1, 1, -1}, {-1, 0, -1}, {-1, -1, 0}, {1, -1, 0},
                                    {1, 1, 0},    {-1, 1, 0},  {-1, -1, 1}, {0, -1, 1},  {1, -1, 1},
                                    {1, 0, 1},    {1, 1, 1},   {0, 1, 1},   {-1, 1, 1},  {-1, 0, 1}};

// gradient of the serendipity shape function of a mid-edge node (one zero coordinate)
void edge_gradient(const signed char p[3], const double x[3], double g[3]) {
  double lin[3];
  for (int d = 0; d < 3; ++d) lin[d] = 1.0 + p[d] * x[d];
  int k = (p[0] == 0) ? 0 : (p[1] == 0 ? 1 : 2);
  int o1 = (k + 1) % 3, o2 = (k + 2) % 3;
  double bub = 1.0 - x[k] * x[k];
  g[k] = 0.25 * (-2.0 * x[k]) * lin[o1] * lin[o2];
  g[o1] = 0.25 * bub * p[o1] * lin[o2];
  g[o2] = 0.25 * bub * lin[o1] * p[o2];
}

void gradients(int nen, const double x[3], double (*g)[3]) {
  for (int a = 0; a < nen; ++a) {
    const signed char* p = (nen == 8) ? kCorner8[a] : kRing20[a];
    bool corner = p[0] != 0 && p[1] != 0 && p[2] != 0;
    if (!corner) { edge_gradient(p, x, g[a]); continue; }
    double lin[3] = {1.0 + p[0] * x[0], 1.0 + p[1] * x[1], 1.0 + p[2] * x[2]};
    if (nen == 8) {
      g[a][0] = 0.125 * p[0] * lin[1] * lin[2];
      g[a][1] = 0.125 * lin[0] * p[1] * lin[2];
      g[a][2] = 0.125 * lin[0] * lin[1] * p[2];
    } else {
      double q = p[0] * x[0] + p[1] * x[1] + p[2] * x[2] - 2.0;
      double prod = lin[0] * lin[1] * lin[2];
      g[a][0] = 0.125 * (p[0] * lin[1] * lin[2] * q + prod * p[0]);
      g[a][1] = 0.125 * (lin[0] * p[1] * lin[2] * q + prod * p[1]);
      g[a][2] = 0.125 * (lin[0] * lin[1] * p[2] * q + prod * p[2]);
    }
  }
}

void matmul(int n, int m, int p, const double* a, const double* b, double* c) {
  for (int j = 0; j < p; ++j)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int k = 0; k < m; ++k) s += a[i + n * k] * b[k + m * j];
      c[i + n * j] = s;
    }
}

// Gauss-Jordan inverse with partial pivoting, column-major, in place.
bool gauss_jordan_inverse(int n, double* a) {
  std::vector<double> aug(2 * n * n, 0.0);  // [A | I], row-major rows of length 2n
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) aug[i * 2 * n + j] = a[i + n * j];
    aug[i * 2 * n + n + i] = 1.0;
  }
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(aug[r * 2 * n + c]) > std::fabs(aug[piv * 2 * n + c])) piv = r;
    if (aug[piv * 2 * n + c] == 0.0) return false;
    if (piv != c)
      for (int j = 0; j < 2 * n; ++j) std::swap(aug[piv * 2 * n + j], aug[c * 2 * n + j]);
    double inv = 1.0 / aug[c * 2 * n + c];
    for (int j = 0; j < 2 * n; ++j) aug[c * 2 * n + j] *= inv;
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      double f = aug[r * 2 * n + c];
      if (f == 0.0) continue;
      for (int j = 0; j < 2 * n; ++j) aug[r * 2 * n + j] -= f * aug[c * 2 * n + j];
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) a[i + n * j] = aug[i * 2 * n + n + j];
  return true;
}

// Rodrigues rotation matrix as written inline at mod_struct_calcmat.f90:556-574
void rotation_matrix(const double n[3], double alpha, double* aa) {
  double c = std::cos(alpha), s = std::sin(alpha), omc = 1.0 - c;
  aa[0 + 3 * 0] = c + n[0] * n[0] * omc;
  aa[1 + 3 * 1] = c + n[1] * n[1] * omc;
  aa[2 + 3 * 2] = c + n[2] * n[2] * omc;
  aa[0 + 3 * 1] = n[0] * n[1] * omc - n[2] * s;
  aa[1 + 3 * 0] = n[0] * n[1] * omc + n[2] * s;
  aa[0 + 3 * 2] = n[0] * n[2] * omc + n[1] * s;
  aa[2 + 3 * 0] = n[0] * n[2] * omc - n[1] * s;
  aa[1 + 3 * 2] = n[1] * n[2] * omc - n[0] * s;
  aa[2 + 3 * 1] = n[1] * n[2] * omc + n[0] * s;
}

// 6x6 Voigt/Mandel transformation of a 3x3 rotation (mod_struct_calcmat.f90:578-589)
void voigt_rotation(const double* aa, double* bb) {
  auto a = [&](int i, int j) { return aa[i + 3 * j]; };  // 0-based
  for (int col = 0; col < 3; ++col) {
    double* b = bb + 6 * col;
    b[0] = a(0, col) * a(0, col); b[1] = a(1, col) * a(1, col); b[2] = a(2, col) * a(2, col);
    b[3] = kSqrt2 * a(1, col) * a(0, col); b[4] = kSqrt2 * a(0, col) * a(2, col); b[5] = kSqrt2 * a(1, col) * a(2, col);
  }
  const int pr[3][2] = {{0, 1}, {0, 2}, {1, 2}};
  for (int q = 0; q < 3; ++q) {
    int i = pr[q][0], j = pr[q][1];
    double* b = bb + 6 * (3 + q);
    b[0] = kSqrt2 * a(0, i) * a(0, j); b[1] = kSqrt2 * a(1, i) * a(1, j); b[2] = kSqrt2 * a(2, i) * a(2, j);
    b[3] = a(1, i) * a(0, j) + a(1, j) * a(0, i);
    b[4] = a(0, i) * a(2, j) + a(0, j) * a(2, i);
    b[5] = a(1, i) * a(2, j) + a(1, j) * a(2, i);
  }
}

void rotate_voigt(const double* aa, const double* ee, double* out) {
  double bb[36], bt[36], tmp[36];
  voigt_rotation(aa, bb);
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) bt[i + 6 * j] = bb[j + 6 * i];
  matmul(6, 6, 6, bt, ee, tmp);
  matmul(6, 6, 6, tmp, bb, out);
}

}  // namespace

void voxel_stiffness(int nen, double nu, double* khat) {
  const int nd = 3 * nen;
  std::fill(khat, khat + nd * nd, 0.0);
  const double lam = nu / ((1 + nu) * (1 - 2 * nu)), mu = 1.0 / (2 * (1 + nu));
  const int ng = (nen == 8) ? 2 : 3;
  double pts[3], wts[3];
  if (ng == 2) { pts[0] = -std::sqrt(1.0 / 3.0); pts[1] = -pts[0]; wts[0] = wts[1] = 1.0; }
  else { pts[0] = -std::sqrt(3.0 / 5.0); pts[1] = 0.0; pts[2] = -pts[0]; wts[0] = wts[2] = 5.0 / 9.0; wts[1] = 8.0 / 9.0; }
  double g[20][3];
  // unit edge: d/dx = 2 d/dxi, dV = dxi/8
  for (int i = 0; i < ng; ++i)
    for (int j = 0; j < ng; ++j)
      for (int k = 0; k < ng; ++k) {
        const double x[3] = {pts[i], pts[j], pts[k]};
        gradients(nen, x, g);
        const double w = wts[i] * wts[j] * wts[k] * 0.125;
        for (int a = 0; a < nen; ++a)
          for (int b = 0; b < nen; ++b) {
            double ga[3] = {2 * g[a][0], 2 * g[a][1], 2 * g[a][2]};
            double gb[3] = {2 * g[b][0], 2 * g[b][1], 2 * g[b][2]};
            double dot = ga[0] * gb[0] + ga[1] * gb[1] + ga[2] * gb[2];
            for (int r = 0; r < 3; ++r)
              for (int c = 0; c < 3; ++c) {
                double v = lam * ga[r] * gb[c] + mu * ga[c] * gb[r] + (r == c ? mu * dot : 0.0);
                khat[(3 * a + r) + nd * (3 * b + c)] += w * v;
              }
          }
      }
}

void macro_shape8(const double xi[3], double N[8]) {
  for (int a = 0; a < 8; ++a) {
    double v = 1.0;
    for (int d = 0; d < 3; ++d) v *= 0.5 * (1.0 + kCorner8[a][d] * xi[d]);
    N[a] = v;
  }
}

void geom_to_xi(const double x[3], const double lo[3], const double hi[3], double xi[3]) {
  for (int d = 0; d < 3; ++d) xi[d] = 2.0 / (hi[d] - lo[d]) * x[d] - (hi[d] + lo[d]) / (hi[d] - lo[d]);
}

void macro_modes(double eps, double* uu) {
  // (load case, component, macro node, multiple of eps) of the nonzero entries
  static const signed char kNZ[][4] = {
      {1, 1, 2, 1}, {1, 1, 3, 1}, {1, 1, 6, 1}, {1, 1, 7, 1},     {2, 2, 3, 1}, {2, 2, 4, 1},
      {2, 2, 7, 1}, {2, 2, 8, 1}, {3, 3, 5, 1}, {3, 3, 6, 1},     {3, 3, 7, 1}, {3, 3, 8, 1},
      {4, 1, 1, 1}, {4, 1, 2, 1}, {4, 1, 5, 1}, {4, 1, 6, 1},     {5, 1, 1, 1}, {5, 1, 2, 1},
      {5, 1, 3, 1}, {5, 1, 4, 1}, {6, 2, 5, 1}, {6, 2, 6, 1},     {6, 2, 7, 1}, {6, 2, 8, 1},
      {7, 1, 8, 1}, {8, 2, 1, 1}, {9, 2, 2, 1}, {10, 3, 1, 1},    {11, 3, 2, 1}, {12, 3, 3, 1},
      {13, 3, 4, 1}, {14, 1, 4, 1}, {15, 1, 5, 1}, {16, 1, 6, 1}, {17, 1, 7, 1}, {18, 1, 8, 1},
      {18, 3, 6, -2}, {19, 2, 1, 1}, {19, 3, 7, -3}, {20, 2, 2, 1}, {20, 3, 8, -4}, {21, 2, 3, 1},
      {22, 2, 4, 1}, {23, 2, 5, 1}, {24, 2, 6, 1}, {24, 2, 7, -1}};
  std::fill(uu, uu + 8 * 3 * 24, 0.0);
  for (const auto& e : kNZ) {
    double v = e[3] == 1 ? eps : (e[3] == -1 ? -eps : e[3] * eps);
    uu[(e[2] - 1) + 8 * (e[1] - 1) + 24 * (e[0] - 1)] = v;
  }
}

double boundary_value(const double* uu, const double N[8], int c, int lc) {
  double s = 0.0;
  for (int l = 0; l < 8; ++l) s += N[l] * uu[l + 8 * c + 24 * lc];
  return s;
}

void macro_shape20(const double xi[3], double N[20]) {
  // ANSYS 20-node brick as phi_NN_hexe20 writes it: corners 1-8, then the mid-edge nodes of
  // the bottom ring (9-12), the top ring (13-16) and the vertical edges (17-20); every product
  // is evaluated left to right as there
  const double f = 1.0 / 8.0, q = 1.0 / 4.0, e = 1.0, z = 2.0;
  const double x = xi[0], y = xi[1], w = xi[2];
  N[0] = f * (e - x) * (e - y) * (e - w) * (-x - y - w - z);
  N[1] = f * (e + x) * (e - y) * (e - w) * (x - y - w - z);
  N[2] = f * (e + x) * (e + y) * (e - w) * (x + y - w - z);
  N[3] = f * (e - x) * (e + y) * (e - w) * (-x + y - w - z);
  N[4] = f * (e - x) * (e - y) * (e + w) * (-x - y + w - z);
  N[5] = f * (e + x) * (e - y) * (e + w) * (x - y + w - z);
  N[6] = f * (e + x) * (e + y) * (e + w) * (x + y + w - z);
  N[7] = f * (e - x) * (e + y) * (e + w) * (-x + y + w - z);
  N[8] = q * (e - x * x) * (e - y) * (e - w);
  N[9] = q * (e + x) * (e - y * y) * (e - w);
  N[10] = q * (e - x * x) * (e + y) * (e - w);
  N[11] = q * (e - x) * (e - y * y) * (e - w);
  N[12] = q * (e - x * x) * (e - y) * (e + w);
  N[13] = q * (e + x) * (e - y * y) * (e + w);
  N[14] = q * (e - x * x) * (e + y) * (e + w);
  N[15] = q * (e - x) * (e - y * y) * (e + w);
  N[16] = q * (e - x) * (e - y) * (e - w * w);
  N[17] = q * (e + x) * (e - y) * (e - w * w);
  N[18] = q * (e + x) * (e + y) * (e - w * w);
  N[19] = q * (e - x) * (e + y) * (e - w * w);
}

namespace {
// Nonzero entries of init_displ_hexe20 (mod_write_deck.f90:118-279) as (load case, component,
// macro node, multiple of eps), all 1-based.  Four entries are written there with default-kind
// (single precision) literals (`.9*eps`, `-.7*eps`): their multiples are those float values.
struct ModeEntry { signed char lc, comp, node; double mult; };
constexpr double F09 = (double)0.9f, F07 = (double)0.7f;
const ModeEntry kModes20[] = {
    {1, 1, 2, 1.0}, {1, 1, 3, 1.0}, {1, 1, 6, 1.0}, {1, 1, 7, 1.0}, {1, 1, 9, 0.5}, {1, 1, 10, 1.0},
    {1, 1, 11, 0.5}, {1, 1, 13, 0.5}, {1, 1, 14, 1.0}, {1, 1, 15, 0.5}, {1, 1, 18, 1.0}, {1, 1, 19, 1.0},
    {2, 2, 3, 1.0}, {2, 2, 4, 1.0}, {2, 2, 7, 1.0}, {2, 2, 8, 1.0}, {2, 2, 10, 0.5}, {2, 2, 11, 1.0},
    {2, 2, 12, 0.5}, {2, 2, 14, 0.5}, {2, 2, 15, 1.0}, {2, 2, 16, 0.5}, {2, 2, 19, 1.0}, {2, 2, 20, 1.0},
    {3, 3, 5, 1.0}, {3, 3, 6, 1.0}, {3, 3, 7, 1.0}, {3, 3, 8, 1.0}, {3, 3, 13, 1.0}, {3, 3, 14, 1.0},
    {3, 3, 15, 1.0}, {3, 3, 16, 1.0}, {3, 3, 17, 0.5}, {3, 3, 18, 0.5}, {3, 3, 19, 0.5}, {3, 3, 20, 0.5},
    {4, 1, 1, 1.0}, {4, 1, 2, 1.0}, {4, 1, 5, 1.0}, {4, 1, 6, 1.0}, {4, 1, 9, 1.0}, {4, 1, 10, 0.5},
    {4, 1, 12, 0.5}, {4, 1, 13, 1.0}, {4, 1, 14, 0.5}, {4, 1, 16, 0.5}, {4, 1, 17, 1.0}, {4, 1, 18, 1.0},
    {5, 1, 1, 1.0}, {5, 1, 2, 1.0}, {5, 1, 3, 1.0}, {5, 1, 4, 1.0}, {5, 1, 9, 1.0}, {5, 1, 10, 1.0},
    {5, 1, 11, 1.0}, {5, 1, 12, 1.0}, {5, 1, 17, 0.5}, {5, 1, 18, 0.5}, {5, 1, 19, 0.5}, {5, 1, 20, 0.5},
    {6, 2, 5, 1.0}, {6, 2, 6, 1.0}, {6, 2, 7, 1.0}, {6, 2, 8, 1.0}, {6, 2, 13, 1.0}, {6, 2, 14, 1.0},
    {6, 2, 15, 1.0}, {6, 2, 16, 1.0}, {6, 2, 17, 0.5}, {6, 2, 18, 0.5}, {6, 2, 19, 0.5}, {6, 2, 20, 0.5},
    {7, 1, 8, 1.0}, {7, 1, 15, 0.5}, {7, 1, 20, 0.5}, {8, 2, 1, -2.0}, {8, 2, 9, 0.5}, {8, 2, 17, 0.5},
    {9, 2, 2, -1.0}, {9, 2, 9, 0.5}, {9, 2, 18, 0.5}, {10, 3, 1, -1.0}, {10, 3, 9, 0.5}, {10, 3, 12, 0.1},
    {10, 3, 17, 0.5}, {11, 3, 2, -2.0}, {11, 3, 10, 0.5}, {11, 3, 18, 0.5}, {12, 3, 11, 0.1}, {12, 3, 19, F09},
    {13, 3, 20, 5.0}, {14, 1, 4, 0.2}, {14, 1, 12, 0.5}, {14, 1, 20, 5.0}, {15, 1, 5, 1.0}, {15, 1, 13, 0.5},
    {16, 1, 6, 5.0}, {16, 1, 18, 0.2}, {17, 1, 14, 0.5}, {17, 1, 19, 0.3}, {18, 1, 15, 0.1}, {18, 1, 20, 0.1},
    {18, 3, 6, -F07}, {18, 3, 13, -0.1}, {18, 3, 14, -1.0}, {19, 2, 9, 0.5}, {19, 2, 12, 0.5}, {19, 2, 17, 0.5},
    {19, 3, 7, -3.0}, {19, 3, 14, -1.5}, {19, 3, 19, -1.5}, {20, 2, 16, 0.1}, {20, 3, 8, -3.0}, {20, 3, 15, -0.1},
    {21, 2, 3, 5.0}, {21, 2, 10, 0.5}, {21, 2, 19, 0.5}, {22, 2, 11, 5.0}, {22, 2, 20, 0.5}, {23, 2, 16, 2.0},
    {24, 2, 13, 5.0}, {24, 2, 19, -0.5}, {25, 3, 9, 2.0}, {26, 3, 10, 5.0}, {27, 2, 11, -0.1}, {27, 3, 11, 1.0},
    {28, 3, 12, 4.0}, {29, 2, 13, 0.1}, {29, 3, 13, -4.0}, {30, 1, 14, -0.1}, {30, 3, 6, 2.0}, {31, 2, 15, -0.1},
    {31, 3, 3, 5.0}, {32, 3, 16, -0.5}, {33, 1, 6, 0.1}, {33, 1, 17, -1.0}, {34, 2, 18, -4.0}, {35, 2, 19, -1.0},
    {36, 2, 20, 2.0}, {37, 1, 1, 3.0}, {38, 2, 2, -5.0}, {39, 1, 3, -3.0}, {40, 2, 4, -2.0}, {41, 1, 5, 5.0},
    {42, 2, 6, 3.0}, {43, 1, 7, -4.0}, {44, 2, 8, 4.0}, {45, 2, 17, 2.0}, {46, 3, 4, -2.0}, {46, 3, 14, -1.5},
    {47, 1, 18, -1.0}, {47, 1, 19, -1.0}, {47, 1, 20, 2.0}, {48, 3, 15, -1.0}, {49, 1, 10, -F09}, {49, 1, 14, -F07},
    {49, 1, 16, 1.0}, {50, 2, 15, 1.0}, {51, 1, 9, 1.0}, {52, 2, 10, 3.0}, {53, 1, 11, -1.0}, {54, 2, 12, 5.0},
    {55, 1, 4, -1.5}, {56, 2, 14, -5.0}, {57, 1, 15, -1.0}, {58, 1, 16, -1.0}, {59, 3, 17, 1.0}, {60, 3, 18, -1.0}};
}  // namespace

void macro_modes20(double eps, double* uu) {
  std::fill(uu, uu + 20 * 3 * 60, 0.0);
  for (const ModeEntry& m : kModes20) uu[(m.node - 1) + 20 * (m.comp - 1) + 60 * (m.lc - 1)] = m.mult * eps;
}

void macro_shape(int order, const double xi[3], double* N) {
  if (order == 2) macro_shape20(xi, N);
  else macro_shape8(xi, N);
}

void macro_modes_of_order(int order, double eps, double* uu) {
  if (order == 2) macro_modes20(eps, uu);
  else macro_modes(eps, uu);
}

double boundary_value_n(int nm, const double* uu, const double* N, int c, int lc) {
  double s = 0.0;
  for (int l = 0; l < nm; ++l) s += N[l] * uu[l + nm * c + 3 * nm * lc];
  return s;
}

void loadcase_matrix(int order, double e, double* vv) {
  const int nm = macro_nodes(order), nl = 3 * nm;
  std::vector<double> uu((size_t)nm * 3 * nl);
  macro_modes_of_order(order, e, uu.data());
  // vv(r, lc) = uu(l, k, lc), r = (k-1)*nm + l: the load-case matrix is the boundary-mode table
  // flattened component-major (exact for init_loadcase_el_order_lin, mod_struct_calcmat.f90:
  // 1684-1770, and for every well-formed entry of init_loadcase_el_order_quad, :1780-2028)
  for (int lc = 0; lc < nl; ++lc)
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < nm; ++l) vv[(nm * k + l) + nl * lc] = uu[l + nm * k + nl * lc];
  if (order == 2) {
    // the two entries the quadratic table writes as 0.9_rk*e where the boundary modes use the
    // single-precision .9*eps: rows 10 and 59 of load cases 49 and 12
    vv[9 + nl * 48] = -0.9 * e;
    vv[58 + nl * 11] = 0.9 * e;
  }
}

double symmetry_deviation(int n, const double* a) {
  double d = 0.0, m = 0.0;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      d = std::max(d, std::fabs(a[i + n * j] - a[j + n * i]));
      m = std::max(m, std::fabs(a[i + n * j]));
    }
  return m > 0.0 ? d / m : 0.0;
}

void homogenise(int order, const double* ff, const int64_t L[3], const double delta[3], double rve_strain,
                dtc_domain_out* out) {
  const int nl = macro_loadcases(order);
  double* ff_out = order == 2 ? out->macro2->ff : out->ff;
  double* km = order == 2 ? out->macro2->kmacro : out->kmacro;
  if (ff_out != ff) std::memcpy(ff_out, ff, sizeof(double) * nl * nl);
  std::vector<double> vv((size_t)nl * nl);
  loadcase_matrix(order, rve_strain, vv.data());
  gauss_jordan_inverse(nl, vv.data());
  matmul(nl, nl, nl, ff, vv.data(), km);
  out->sym_k = symmetry_deviation(nl, km);
  const double X = (double)L[0] * delta[0], Y = (double)L[1] * delta[1], Z = (double)L[2] * delta[2];
  auto f = [&](int r, int c) { return ff[(r - 1) + nl * c]; };  // r 1-based, c 0-based
  double fv[36];
  if (order == 2) {
    for (int c = 0; c < 6; ++c) {  // mod_struct_calcmat.f90:368-401: the 8 nodes of each face
      fv[0 + 6 * c] = (f(2, c) + f(3, c) + f(6, c) + f(7, c) + f(10, c) + f(14, c) + f(18, c) + f(19, c)) / (Y * Z);
      fv[1 + 6 * c] = (f(23, c) + f(24, c) + f(27, c) + f(28, c) + f(31, c) + f(35, c) + f(39, c) + f(40, c)) / (X * Z);
      fv[2 + 6 * c] = (f(45, c) + f(46, c) + f(47, c) + f(48, c) + f(53, c) + f(54, c) + f(55, c) + f(56, c)) / (X * Y);
      fv[3 + 6 * c] =
          0.5 * ((f(3, c) + f(4, c) + f(7, c) + f(8, c) + f(11, c) + f(15, c) + f(19, c) + f(20, c)) / (X * Z) +
                 (f(22, c) + f(23, c) + f(26, c) + f(27, c) + f(30, c) + f(34, c) + f(38, c) + f(39, c)) / (Y * Z));
      fv[4 + 6 * c] =
          0.5 * ((f(5, c) + f(6, c) + f(7, c) + f(8, c) + f(13, c) + f(14, c) + f(15, c) + f(16, c)) / (X * Y) +
                 (f(42, c) + f(43, c) + f(46, c) + f(47, c) + f(50, c) + f(54, c) + f(58, c) + f(59, c)) / (Y * Z));
      fv[5 + 6 * c] =
          0.5 * ((f(25, c) + f(26, c) + f(27, c) + f(28, c) + f(33, c) + f(34, c) + f(35, c) + f(36, c)) / (X * Y) +
                 (f(43, c) + f(44, c) + f(47, c) + f(48, c) + f(51, c) + f(55, c) + f(59, c) + f(60, c)) / (X * Z));
    }
  } else {
    for (int c = 0; c < 6; ++c) {  // mod_struct_calcmat.f90:345-359
      fv[0 + 6 * c] = (f(2, c) + f(3, c) + f(6, c) + f(7, c)) / (Y * Z);
      fv[1 + 6 * c] = (f(11, c) + f(12, c) + f(15, c) + f(16, c)) / (X * Z);
      fv[2 + 6 * c] = (f(21, c) + f(22, c) + f(23, c) + f(24, c)) / (X * Y);
      fv[3 + 6 * c] = 0.5 * ((f(3, c) + f(4, c) + f(7, c) + f(8, c)) / (X * Z) + (f(10, c) + f(11, c) + f(14, c) + f(15, c)) / (Y * Z));
      fv[4 + 6 * c] = 0.5 * ((f(5, c) + f(6, c) + f(7, c) + f(8, c)) / (X * Y) + (f(18, c) + f(19, c) + f(22, c) + f(23, c)) / (Y * Z));
      fv[5 + 6 * c] = 0.5 * ((f(13, c) + f(14, c) + f(15, c) + f(16, c)) / (X * Y) + (f(19, c) + f(20, c) + f(23, c) + f(24, c)) / (X * Z));
    }
  }
  // C = fv * meps, meps = diag(1e6, 1e6, 1e6, -1e6, -1e6, 1e6) (:434-439)
  const double meps[6] = {1e6, 1e6, 1e6, -1e6, -1e6, 1e6};
  for (int j = 0; j < 6; ++j)
    for (int i = 0; i < 6; ++i) out->c[i + 6 * j] = fv[i + 6 * j] * meps[j];
  out->sym_c = symmetry_deviation(6, out->c);
  for (int j = 0; j < 6; ++j)
    for (int i = 0; i < 6; ++i) out->ee[i + 6 * j] = (out->c[i + 6 * j] + out->c[j + 6 * i]) / 2.0;
  out->sym_ee = symmetry_deviation(6, out->ee);
}

void energy_to_ff(int order, const double* gram, double* ff) {
  const int nm = macro_nodes(order), nl = macro_loadcases(order);
  // the load-case matrix of the modes actually prescribed (eps = 1e-6, mod_write_deck.f90:61)
  std::vector<double> uu((size_t)nm * 3 * nl), vv((size_t)nl * nl);
  macro_modes_of_order(order, 1e-6, uu.data());
  for (int lc = 0; lc < nl; ++lc)
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < nm; ++l) vv[(nm * k + l) + (size_t)nl * lc] = uu[l + nm * k + (size_t)nl * lc];
  gauss_jordan_inverse(nl, vv.data());
  for (int lc = 0; lc < nl; ++lc)
    for (int r = 0; r < nl; ++r) {
      double s = 0.0;
      for (int a = 0; a < nl; ++a) s += vv[a + (size_t)nl * r] * gram[a + (size_t)nl * lc];
      ff[r + (size_t)nl * lc] = s;
    }
}

void finish_rotation(const double ee[36], int which, const int64_t ang[3], int jj, double crit,
                     dtc_domain_out* out) {
  // quirk kept: the final angle scale is pi / (180 (10^jj - 1)) (:1017, :1464)
  const double scale = kPi / (180.0 * (std::pow(10.0, jj) - 1.0));
  const double alpha0 = (double)ang[0] * scale, phi = (double)ang[1] * scale, eta = (double)ang[2] * scale;
  double n[3] = {std::cos(phi) * std::sin(eta), std::sin(phi) * std::sin(eta), std::cos(eta)};
  const double nrm = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  for (double& v : n) v /= nrm;
  double aa[9], rot[36];
  rotation_matrix(n, alpha0, aa);
  rotate_voigt(aa, ee, rot);
  double alpha = alpha0, nfix[3] = {n[0], n[1], n[2]};
  // axis permutation so that E11 <= E22 <= E33 (:1046-1134)
  auto turn_about_column = [&](int col) {
    double axis[3] = {aa[0 + 3 * col], aa[1 + 3 * col], aa[2 + 3 * col]};
    double r[9], t[9];
    rotation_matrix(axis, kPi / 2, r);
    matmul(3, 3, 3, r, aa, t);
    std::memcpy(aa, t, sizeof(t));
    std::memcpy(nfix, axis, sizeof(axis));
    alpha = kPi / 2;
  };
  const double e1 = rot[0], e2 = rot[7], e3 = rot[14];
  if (e1 < e2 && e1 < e3 && e2 > e3) turn_about_column(0);                              // 132
  else if (e1 < e2 && e1 > e3 && e2 > e3) { turn_about_column(1); turn_about_column(0); } // 231
  else if (e1 > e2 && e1 < e3 && e2 < e3) turn_about_column(2);                         // 213
  else if (e1 > e2 && e1 > e3 && e2 < e3) { turn_about_column(2); turn_about_column(0); } // 312
  else if (e1 > e2 && e1 > e3 && e2 > e3) turn_about_column(1);                         // 321
  rotate_voigt(aa, ee, rot);
  if (which == 1) {  // CR1 records the angle and axis found by the search (:1037-1049)
    out->cr1_angle = alpha0;
    std::memcpy(out->cr1_n, n, sizeof(n));
    std::memcpy(out->cr1_aa, aa, sizeof(aa));
    std::memcpy(out->cr1_ee, rot, sizeof(rot));
    out->cr1_crit = crit;
    out->cr1_iters = jj;
  } else {           // CR2 records them after the permutation (:1583-1597)
    out->cr2_angle = alpha;
    std::memcpy(out->cr2_n, nfix, sizeof(nfix));
    std::memcpy(out->cr2_aa, aa, sizeof(aa));
    std::memcpy(out->cr2_ee, rot, sizeof(rot));
    out->cr2_crit = crit;
    out->cr2_iters = jj;
  }
}

// cos and sin of k degrees, k = 0..180, correctly rounded (ddmath.h), as the device
// computes the refinement levels
void degree_tables(double* c, double* s) {
  for (int k = 0; k <= 180; ++k) {
    double a = (double)k * kPiDiv180;
    dd::sincos_cr(a, &s[k], &c[k]);
  }
}

}  // namespace dtc
