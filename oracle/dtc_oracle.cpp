// dtc_oracle.cpp -- TEST INFRASTRUCTURE ONLY (see dtc_oracle.h).
//
// CPU FP64 restatement of the reference's per-domain path.  Every function cites the
// reference file:line it follows.  Compiled with -ffp-contract=off so that each
// expression is evaluated in the written order without fused multiply-adds.
#include "dtc_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <quadmath.h>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// geb-lib constants (the submodule is absent; values as mod_tensor_opt.f90:61-62 states them)
const double kPi = std::acos(-1.0);
const double kPiDiv180 = kPi / 180.0;
const double kSq2 = std::sqrt(2.0);
const double kNumZero = 1.0e-9;
const double kDeltaB = 1.0e-9;   // mod_write_deck.f90:9
const double kEpsBC = 1.0e-6;    // mod_write_deck.f90:61 (hard-coded boundary displacement)

// ---------------------------------------------------------------------------------------
// Boundary modes uu(l,c,lc) = f * eps (mod_write_deck.f90:63-116), 24 load cases of the
// linear macro element.  One entry per nonzero: load case, component, macro node, factor.
struct ModeNZ { int lc, comp, node; double f; };
const ModeNZ kModes[] = {
    {1, 1, 2, 1}, {1, 1, 3, 1}, {1, 1, 6, 1}, {1, 1, 7, 1},
    {2, 2, 3, 1}, {2, 2, 4, 1}, {2, 2, 7, 1}, {2, 2, 8, 1},
    {3, 3, 5, 1}, {3, 3, 6, 1}, {3, 3, 7, 1}, {3, 3, 8, 1},
    {4, 1, 1, 1}, {4, 1, 2, 1}, {4, 1, 5, 1}, {4, 1, 6, 1},
    {5, 1, 1, 1}, {5, 1, 2, 1}, {5, 1, 3, 1}, {5, 1, 4, 1},
    {6, 2, 5, 1}, {6, 2, 6, 1}, {6, 2, 7, 1}, {6, 2, 8, 1},
    {7, 1, 8, 1}, {8, 2, 1, 1}, {9, 2, 2, 1}, {10, 3, 1, 1}, {11, 3, 2, 1},
    {12, 3, 3, 1}, {13, 3, 4, 1}, {14, 1, 4, 1}, {15, 1, 5, 1}, {16, 1, 6, 1},
    {17, 1, 7, 1}, {18, 1, 8, 1}, {18, 3, 6, -2}, {19, 2, 1, 1}, {19, 3, 7, -3},
    {20, 2, 2, 1}, {20, 3, 8, -4}, {21, 2, 3, 1}, {22, 2, 4, 1}, {23, 2, 5, 1},
    {24, 2, 6, 1}, {24, 2, 7, -1},
};

void boundary_modes(double eps, double* uu) {  // uu(8,3,24) column-major
  std::fill(uu, uu + 8 * 3 * 24, 0.0);
  for (const ModeNZ& m : kModes) {
    double v = (m.f == 1) ? eps : ((m.f == -1) ? -eps : m.f * eps);
    uu[(m.node - 1) + 8 * (m.comp - 1) + 24 * (m.lc - 1)] = v;
  }
}

// vv(r, lc) = uu(l, k, lc) with r = (k-1)*8 + l: the load-case matrix of
// mod_struct_calcmat.f90:1684-1770 is the component-major flattening of uu.
void loadcase_matrix(double eps, double* vv) {
  std::vector<double> uu(8 * 3 * 24);
  boundary_modes(eps, uu.data());
  for (int lc = 0; lc < 24; ++lc)
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < 8; ++l) vv[(k * 8 + l) + 24 * lc] = uu[l + 8 * k + 24 * lc];
}

// Boundary modes of the quadratic macro element, init_displ_hexe20 (mod_write_deck.f90:
// 118-279): one row per statement `uu(:,c,lc) = [20 values]` of the source, values in units
// of eps.  S9 / S7 are the default-kind (single precision) literals `.9` and `.7` the source
// multiplies eps by in four places.
const double S9 = (double)0.9f, S7 = (double)0.7f;
struct Mode20Row { int lc, comp; double f[20]; };
const Mode20Row kModes20[] = {
    {1, 1, {0, 1, 1, 0, 0, 1, 1, 0, .5, 1, .5, 0, .5, 1, .5, 0, 0, 1, 1, 0}},
    {2, 2, {0, 0, 1, 1, 0, 0, 1, 1, 0, .5, 1, .5, 0, .5, 1, .5, 0, 0, 1, 1}},
    {3, 3, {0, 0, 0, 0, 1, 1, 1, 1, 0, 0, 0, 0, 1, 1, 1, 1, .5, .5, .5, .5}},
    {4, 1, {1, 1, 0, 0, 1, 1, 0, 0, 1, .5, 0, .5, 1, .5, 0, .5, 1, 1, 0, 0}},
    {5, 1, {1, 1, 1, 1, 0, 0, 0, 0, 1, 1, 1, 1, 0, 0, 0, 0, .5, .5, .5, .5}},
    {6, 2, {0, 0, 0, 0, 1, 1, 1, 1, 0, 0, 0, 0, 1, 1, 1, 1, .5, .5, .5, .5}},
    {7, 1, {0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, .5, 0, 0, 0, 0, .5}},
    {8, 2, {-2, 0, 0, 0, 0, 0, 0, 0, .5, 0, 0, 0, 0, 0, 0, 0, .5, 0, 0, 0}},
    {9, 2, {0, -1, 0, 0, 0, 0, 0, 0, .5, 0, 0, 0, 0, 0, 0, 0, 0, .5, 0, 0}},
    {10, 3, {-1, 0, 0, 0, 0, 0, 0, 0, .5, 0, 0, .1, 0, 0, 0, 0, .5, 0, 0, 0}},
    {11, 3, {0, -2, 0, 0, 0, 0, 0, 0, 0, .5, 0, 0, 0, 0, 0, 0, 0, .5, 0, 0}},
    {12, 3, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, .1, 0, 0, 0, 0, 0, 0, 0, S9, 0}},
    {13, 3, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 5}},
    {14, 1, {0, 0, 0, .2, 0, 0, 0, 0, 0, 0, 0, .5, 0, 0, 0, 0, 0, 0, 0, 5}},
    {15, 1, {0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, .5, 0, 0, 0, 0, 0, 0, 0}},
    {16, 1, {0, 0, 0, 0, 0, 5, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, .2, 0, 0}},
    {17, 1, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, .5, 0, 0, 0, 0, .3, 0}},
    {18, 1, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, .1, 0, 0, 0, 0, .1}},
    {18, 3, {0, 0, 0, 0, 0, -S7, 0, 0, 0, 0, 0, 0, -.1, -1, 0, 0, 0, 0, 0, 0}},
    {19, 2, {0, 0, 0, 0, 0, 0, 0, 0, .5, 0, 0, .5, 0, 0, 0, 0, .5, 0, 0, 0}},
    {19, 3, {0, 0, 0, 0, 0, 0, -3, 0, 0, 0, 0, 0, 0, -1.5, 0, 0, 0, 0, -1.5, 0}},
    {20, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, .1, 0, 0, 0, 0}},
    {20, 3, {0, 0, 0, 0, 0, 0, 0, -3, 0, 0, 0, 0, 0, 0, -.1, 0, 0, 0, 0, 0}},
    {21, 2, {0, 0, 5, 0, 0, 0, 0, 0, 0, .5, 0, 0, 0, 0, 0, 0, 0, 0, .5, 0}},
    {22, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 5, 0, 0, 0, 0, 0, 0, 0, 0, .5}},
    {23, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 2, 0, 0, 0, 0}},
    {24, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 5, 0, 0, 0, 0, 0, -.5, 0}},
    {25, 3, {0, 0, 0, 0, 0, 0, 0, 0, 2, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {26, 3, {0, 0, 0, 0, 0, 0, 0, 0, 0, 5, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {27, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -.1, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {27, 3, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {28, 3, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 4, 0, 0, 0, 0, 0, 0, 0, 0}},
    {29, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, .1, 0, 0, 0, 0, 0, 0, 0}},
    {29, 3, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -4, 0, 0, 0, 0, 0, 0, 0}},
    {30, 1, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -.1, 0, 0, 0, 0, 0, 0}},
    {30, 3, {0, 0, 0, 0, 0, 2, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {31, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -.1, 0, 0, 0, 0, 0}},
    {31, 3, {0, 0, 5, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {32, 3, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -.5, 0, 0, 0, 0}},
    {33, 1, {0, 0, 0, 0, 0, .1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 0, 0, 0}},
    {34, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -4, 0, 0}},
    {35, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 0}},
    {36, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 2}},
    {37, 1, {3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {38, 2, {0, -5, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {39, 1, {0, 0, -3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {40, 2, {0, 0, 0, -2, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {41, 1, {0, 0, 0, 0, 5, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {42, 2, {0, 0, 0, 0, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {43, 1, {0, 0, 0, 0, 0, 0, -4, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {44, 2, {0, 0, 0, 0, 0, 0, 0, 4, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {45, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 2, 0, 0, 0}},
    {46, 3, {0, 0, 0, -2, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1.5, 0, 0, 0, 0, 0, 0}},
    {47, 1, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, -1, 2}},
    {48, 3, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 0, 0, 0, 0, 0}},
    {49, 1, {0, 0, 0, 0, 0, 0, 0, 0, 0, -S9, 0, 0, 0, -S7, 0, 1, 0, 0, 0, 0}},
    {50, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0}},
    {51, 1, {0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {52, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 3, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {53, 1, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {54, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 5, 0, 0, 0, 0, 0, 0, 0, 0}},
    {55, 1, {0, 0, 0, -1.5, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0}},
    {56, 2, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -5, 0, 0, 0, 0, 0, 0}},
    {57, 1, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 0, 0, 0, 0, 0}},
    {58, 1, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 0, 0, 0, 0}},
    {59, 3, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0}},
    {60, 3, {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, -1, 0, 0}},
};

void boundary_modes20(double eps, double* uu) {  // uu(20,3,60) column-major
  std::fill(uu, uu + 20 * 3 * 60, 0.0);
  for (const Mode20Row& m : kModes20)
    for (int l = 0; l < 20; ++l)
      uu[l + 20 * (m.comp - 1) + 60 * (m.lc - 1)] = m.f[l] == 0 ? 0.0 : m.f[l] * eps;
}

// init_loadcase_el_order_quad (mod_struct_calcmat.f90:1780-2028), vv(60,60).  The source table
// is not usable as written: its row 49 is labelled 59 (so vv(49,:) stays zero and vv is
// singular), 22 entries lack the factor e, and row 54 has 61 values.  Every other entry
// equals the component-major flattening of the boundary modes for eps = e, except two that
// the table writes with the double literal 0.9_rk where the modes use the single-precision .9
// (row 10 of load case 49, row 59 of load case 12).  The oracle uses that flattening with the
// two double entries, i.e. the table with its defects repaired.
void loadcase_matrix_quad(double e, double* vv) {
  std::vector<double> uu(20 * 3 * 60);
  boundary_modes20(e, uu.data());
  for (int lc = 0; lc < 60; ++lc)
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < 20; ++l) vv[(k * 20 + l) + 60 * lc] = uu[l + 20 * k + 60 * lc];
  vv[9 + 60 * 48] = -0.9 * e;
  vv[58 + 60 * 11] = 0.9 * e;
}

// ---------------------------------------------------------------------------------------
// Shape functions and the geometry -> xi map (mod_linfe.f90:19-84)
inline double g1(double xi) { return 0.5 * (1.0 - xi); }
inline double g2(double xi) { return 0.5 * (1.0 + xi); }
inline void phi_nn_hexe8(const double xi[3], double N[8]) {
  N[0] = g1(xi[0]) * g1(xi[1]) * g1(xi[2]);
  N[1] = g2(xi[0]) * g1(xi[1]) * g1(xi[2]);
  N[2] = g2(xi[0]) * g2(xi[1]) * g1(xi[2]);
  N[3] = g1(xi[0]) * g2(xi[1]) * g1(xi[2]);
  N[4] = g1(xi[0]) * g1(xi[1]) * g2(xi[2]);
  N[5] = g2(xi[0]) * g1(xi[1]) * g2(xi[2]);
  N[6] = g2(xi[0]) * g2(xi[1]) * g2(xi[2]);
  N[7] = g1(xi[0]) * g2(xi[1]) * g2(xi[2]);
}
// phi_NN_hexe20 (mod_linfe.f90:827-888): ANSYS 20-node brick, products left to right
inline void phi_nn_hexe20(const double xi[3], double N[20]) {
  const double f = 1. / 8., ff = 1. / 4., e = 1., z = 2.;
  N[0] = f * (e - xi[0]) * (e - xi[1]) * (e - xi[2]) * (-xi[0] - xi[1] - xi[2] - z);
  N[1] = f * (e + xi[0]) * (e - xi[1]) * (e - xi[2]) * (xi[0] - xi[1] - xi[2] - z);
  N[2] = f * (e + xi[0]) * (e + xi[1]) * (e - xi[2]) * (xi[0] + xi[1] - xi[2] - z);
  N[3] = f * (e - xi[0]) * (e + xi[1]) * (e - xi[2]) * (-xi[0] + xi[1] - xi[2] - z);
  N[4] = f * (e - xi[0]) * (e - xi[1]) * (e + xi[2]) * (-xi[0] - xi[1] + xi[2] - z);
  N[5] = f * (e + xi[0]) * (e - xi[1]) * (e + xi[2]) * (xi[0] - xi[1] + xi[2] - z);
  N[6] = f * (e + xi[0]) * (e + xi[1]) * (e + xi[2]) * (xi[0] + xi[1] + xi[2] - z);
  N[7] = f * (e - xi[0]) * (e + xi[1]) * (e + xi[2]) * (-xi[0] + xi[1] + xi[2] - z);
  N[8] = ff * (e - xi[0] * xi[0]) * (e - xi[1]) * (e - xi[2]);
  N[9] = ff * (e + xi[0]) * (e - xi[1] * xi[1]) * (e - xi[2]);
  N[10] = ff * (e - xi[0] * xi[0]) * (e + xi[1]) * (e - xi[2]);
  N[11] = ff * (e - xi[0]) * (e - xi[1] * xi[1]) * (e - xi[2]);
  N[12] = ff * (e - xi[0] * xi[0]) * (e - xi[1]) * (e + xi[2]);
  N[13] = ff * (e + xi[0]) * (e - xi[1] * xi[1]) * (e + xi[2]);
  N[14] = ff * (e - xi[0] * xi[0]) * (e + xi[1]) * (e + xi[2]);
  N[15] = ff * (e - xi[0]) * (e - xi[1] * xi[1]) * (e + xi[2]);
  N[16] = ff * (e - xi[0]) * (e - xi[1]) * (e - xi[2] * xi[2]);
  N[17] = ff * (e + xi[0]) * (e - xi[1]) * (e - xi[2] * xi[2]);
  N[18] = ff * (e + xi[0]) * (e + xi[1]) * (e - xi[2] * xi[2]);
  N[19] = ff * (e - xi[0]) * (e + xi[1]) * (e - xi[2] * xi[2]);
}
inline void phi_nn_macro(int nm, const double xi[3], double* N) {
  if (nm == 20) phi_nn_hexe20(xi, N);
  else phi_nn_hexe8(xi, N);
}
inline void t_geom_xi(const double node[3], const double xa[3], const double xe[3], double t[3]) {
  for (int d = 0; d < 3; ++d) t[d] = 2.0 / (xe[d] - xa[d]) * node[d] - (xe[d] + xa[d]) / (xe[d] - xa[d]);
}

// ---------------------------------------------------------------------------------------
// Element stiffness by Gauss quadrature.  Equals the tabulated Hexe08 / Hexe20 of
// mod_linfe.f90:161-776 / 890-4509 times their factor E*a/(144(2nu^2+nu-1)) /
// E*a/(256(2nu^2+nu-1)) with a = phdsize*delta (checked against tests/golden).
// Local node order: HEX08 = mod_gen_quadmesh.f90:298-306, HEX20 = the "ring" order of
// mod_gen_quadmesh.f90:244-265 (corner, mid-edge, corner, ... per face ring).
const int kHex08Xi[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                            {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
const int kHex20Xi[20][3] = {{-1, -1, -1}, {0, -1, -1}, {1, -1, -1}, {1, 0, -1}, {1, 1, -1},
                             {0, 1, -1},   {-1, 1, -1}, {-1, 0, -1}, {-1, -1, 0}, {1, -1, 0},
                             {1, 1, 0},    {-1, 1, 0},  {-1, -1, 1}, {0, -1, 1},  {1, -1, 1},
                             {1, 0, 1},    {1, 1, 1},   {0, 1, 1},   {-1, 1, 1},  {-1, 0, 1}};

void shape_grad(int nen, const double x[3], double dN[][3]) {
  if (nen == 8) {
    for (int a = 0; a < 8; ++a) {
      const int* p = kHex08Xi[a];
      double f0 = 1 + p[0] * x[0], f1 = 1 + p[1] * x[1], f2 = 1 + p[2] * x[2];
      dN[a][0] = 0.125 * p[0] * f1 * f2;
      dN[a][1] = 0.125 * f0 * p[1] * f2;
      dN[a][2] = 0.125 * f0 * f1 * p[2];
    }
    return;
  }
  for (int a = 0; a < 20; ++a) {
    const int* p = kHex20Xi[a];
    int nz = (p[0] != 0) + (p[1] != 0) + (p[2] != 0);
    if (nz == 3) {
      double f[3] = {1 + p[0] * x[0], 1 + p[1] * x[1], 1 + p[2] * x[2]};
      double s = p[0] * x[0] + p[1] * x[1] + p[2] * x[2] - 2.0;
      for (int d = 0; d < 3; ++d) {
        int e1 = (d + 1) % 3, e2 = (d + 2) % 3;
        dN[a][d] = 0.125 * (p[d] * f[e1] * f[e2] * s + f[0] * f[1] * f[2] * p[d]);
      }
    } else {
      int k = (p[0] == 0) ? 0 : ((p[1] == 0) ? 1 : 2);
      int o1 = (k + 1) % 3, o2 = (k + 2) % 3;
      double q = 1 - x[k] * x[k];
      double f1 = 1 + p[o1] * x[o1], f2 = 1 + p[o2] * x[o2];
      dN[a][k] = 0.25 * (-2.0 * x[k]) * f1 * f2;
      dN[a][o1] = 0.25 * q * p[o1] * f2;
      dN[a][o2] = 0.25 * q * f1 * p[o2];
    }
  }
}

void element_stiffness(int nen, double E, double a, double nu, double* ke) {
  const int nd = 3 * nen;
  std::fill(ke, ke + nd * nd, 0.0);
  double lam = E * nu / ((1 + nu) * (1 - 2 * nu)), mu = E / (2 * (1 + nu));
  int ng = (nen == 8) ? 2 : 3;
  double gp[3], gw[3];
  if (ng == 2) { gp[0] = -1 / std::sqrt(3.0); gp[1] = -gp[0]; gw[0] = gw[1] = 1; }
  else { gp[0] = -std::sqrt(0.6); gp[1] = 0; gp[2] = std::sqrt(0.6); gw[0] = gw[2] = 5.0 / 9; gw[1] = 8.0 / 9; }
  double dN[20][3];
  std::vector<double> B(6 * nd);
  for (int i = 0; i < ng; ++i)
    for (int j = 0; j < ng; ++j)
      for (int k = 0; k < ng; ++k) {
        double x[3] = {gp[i], gp[j], gp[k]};
        shape_grad(nen, x, dN);
        std::fill(B.begin(), B.end(), 0.0);
        for (int n = 0; n < nen; ++n) {
          double dx = dN[n][0] * 2 / a, dy = dN[n][1] * 2 / a, dz = dN[n][2] * 2 / a;
          B[0 * nd + 3 * n] = dx; B[1 * nd + 3 * n + 1] = dy; B[2 * nd + 3 * n + 2] = dz;
          B[3 * nd + 3 * n] = dy; B[3 * nd + 3 * n + 1] = dx;
          B[4 * nd + 3 * n + 1] = dz; B[4 * nd + 3 * n + 2] = dy;
          B[5 * nd + 3 * n] = dz; B[5 * nd + 3 * n + 2] = dx;
        }
        double w = gw[i] * gw[j] * gw[k] * (a / 2) * (a / 2) * (a / 2);
        for (int r = 0; r < nd; ++r)
          for (int c = 0; c < nd; ++c) {
            const double* br = &B[0];
            double ex = B[0 * nd + r], ey = B[1 * nd + r], ez = B[2 * nd + r];
            double sx = (lam + 2 * mu) * B[0 * nd + c] + lam * B[1 * nd + c] + lam * B[2 * nd + c];
            double sy = lam * B[0 * nd + c] + (lam + 2 * mu) * B[1 * nd + c] + lam * B[2 * nd + c];
            double sz = lam * B[0 * nd + c] + lam * B[1 * nd + c] + (lam + 2 * mu) * B[2 * nd + c];
            double v = ex * sx + ey * sy + ez * sz + mu * (B[3 * nd + r] * B[3 * nd + c] +
                                                           B[4 * nd + r] * B[4 * nd + c] +
                                                           B[5 * nd + r] * B[5 * nd + c]);
            (void)br;
            ke[r + nd * c] += w * v;
          }
      }
}

// ---------------------------------------------------------------------------------------
// Mesher: literal restatement of gen_quadmesh_from_phi (mod_gen_quadmesh.f90:22-679).
struct Mesh {
  int64_t ne = 0, nn = 0;
  std::vector<int64_t> elems;  // nen*ne, 1-based node ids, 0 = dropped
  std::vector<int64_t> evox;   // voxel index of each element (bookkeeping only)
  std::vector<double> nodes;   // 3*nn
};

bool gen_quadmesh(const orc_domain_in& in, Mesh& m) {
  const int64_t L0 = in.L[0], L1 = in.L[1], L2 = in.L[2];
  const int nen = in.nen;
  int64_t maxv = INT64_MIN;
  for (int64_t i = 0; i < L0 * L1 * L2; ++i) maxv = std::max<int64_t>(maxv, in.phi[i]);
  if (maxv < in.llimit) return false;  // :142-164
  int64_t xdn[3];
  for (int d = 0; d < 3; ++d) xdn[d] = (nen == 8) ? in.L[d] + 1 : 2 * in.L[d] + 1;
  const int64_t ub = xdn[0] * xdn[1] * xdn[2];
  std::vector<int64_t> nodes_no(ub + 1, 0);
  std::vector<int64_t> elems;
  std::vector<int64_t> evox;
  elems.reserve(nen * L0 * L1 * L2);
  const int64_t s1 = xdn[0], s2 = xdn[0] * xdn[1];
  // element generation, x fastest (:226-316)
  for (int64_t kk = 1; kk <= L2; ++kk)
    for (int64_t jj = 1; jj <= L1; ++jj)
      for (int64_t ii = 1; ii <= L0; ++ii) {
        int64_t v = (ii - 1) + L0 * ((jj - 1) + L1 * (kk - 1));
        if (in.phi[v] < in.llimit) continue;
        int64_t el[20];
        if (nen == 8) {
          for (int a = 0; a < 8; ++a) {
            int64_t ox = (kHex08Xi[a][0] + 1) / 2, oy = (kHex08Xi[a][1] + 1) / 2, oz = (kHex08Xi[a][2] + 1) / 2;
            el[a] = (ii - 1 + ox) + (jj - 1 + oy) * s1 + (kk - 1 + oz) * s2;
          }
        } else {
          for (int a = 0; a < 20; ++a) {
            int64_t ox = kHex20Xi[a][0] + 1, oy = kHex20Xi[a][1] + 1, oz = kHex20Xi[a][2] + 1;
            el[a] = (2 * ii - 2 + ox) + (2 * jj - 2 + oy) * s1 + (2 * kk - 2 + oz) * s2;
          }
        }
        for (int a = 0; a < nen; ++a) { nodes_no[el[a]] = -1; elems.push_back(el[a]); }
        evox.push_back(v);
      }
  int64_t ne = (int64_t)evox.size();
  // node numbering by first appearance (:322-341)
  int64_t nn = 0;
  for (int64_t e = 0; e < ne; ++e)
    for (int a = 0; a < nen; ++a)
      if (nodes_no[elems[e * nen + a]] == -1) nodes_no[elems[e * nen + a]] = ++nn;
  for (int64_t e = 0; e < ne * nen; ++e) elems[e] = nodes_no[elems[e]];
  // coordinates (:346-384)
  std::vector<double> nodes(3 * nn);
  for (int64_t ll = 0; ll <= ub; ++ll) {
    if (nodes_no[ll] == 0) continue;
    int64_t kk = ll / s2, jj = (ll - kk * s2) / s1, ii = ll - kk * s2 - jj * s1;
    int64_t id = nodes_no[ll];
    if (nen == 20) {
      nodes[3 * (id - 1) + 2] = ((double)kk / 2.0 + (double)(in.xa_n[2] - 1)) * in.delta[2];
      nodes[3 * (id - 1) + 1] = ((double)jj / 2.0 + (double)(in.xa_n[1] - 1)) * in.delta[1];
      nodes[3 * (id - 1) + 0] = ((double)ii / 2.0 + (double)(in.xa_n[0] - 1)) * in.delta[0];
    } else {
      nodes[3 * (id - 1) + 2] = (double)(kk + in.xa_n[2] - 1) * in.delta[2];
      nodes[3 * (id - 1) + 1] = (double)(jj + in.xa_n[1] - 1) * in.delta[1];
      nodes[3 * (id - 1) + 0] = (double)(ii + in.xa_n[0] - 1) * in.delta[0];
    }
  }
  // colour nodes by max-label propagation over elements (:408-433)
  std::vector<int64_t> node_col(nn + 1);
  for (int64_t i = 1; i <= nn; ++i) node_col[i] = i;
  bool change = true;
  while (change) {
    change = false;
    for (int64_t e = 0; e < ne; ++e) {
      int64_t mn = INT64_MAX, mx = INT64_MIN;
      for (int a = 0; a < nen; ++a) {
        int64_t c = node_col[elems[e * nen + a]];
        mn = std::min(mn, c); mx = std::max(mx, c);
      }
      if (mn != mx) {
        for (int a = 0; a < nen; ++a) node_col[elems[e * nen + a]] = mx;
        change = true;
      }
    }
  }
  std::vector<int64_t> elem_col(ne + 1);
  for (int64_t e = 0; e < ne; ++e) elem_col[e + 1] = node_col[elems[e * nen]];
  // colour list in order of first appearance over nodes (:445-481)
  std::vector<int64_t> colors;
  std::vector<char> tb;
  colors.push_back(node_col[1]);
  for (int64_t i = 1; i <= nn; ++i) {
    if (node_col[i] != colors.back() &&
        std::find(colors.begin(), colors.end(), node_col[i]) == colors.end())
      colors.push_back(node_col[i]);
  }
  tb.assign(colors.size(), 0);
  double xmin[3], xmax[3];
  for (int d = 0; d < 3; ++d) {
    xmin[d] = INFINITY; xmax[d] = -INFINITY;
    for (int64_t i = 0; i < nn; ++i) {
      xmin[d] = std::min(xmin[d], nodes[3 * i + d]);
      xmax[d] = std::max(xmax[d], nodes[3 * i + d]);
    }
  }
  // first region: signed differences without abs (:494-521) -- always true via x_max
  for (int64_t i = 1; i <= nn; ++i) {
    if (node_col[i] != colors[0]) continue;
    const double* x = &nodes[3 * (i - 1)];
    bool hit = false;
    for (int d = 0; d < 3 && !hit; ++d)
      hit = ((x[d] - xmin[d]) < 0.1 * in.delta[d]) || ((x[d] - xmax[d]) < 0.1 * in.delta[d]);
    if (hit) { tb[0] = 1; break; }
  }
  // other regions: |x - bbox face| < 0.1 delta against the mesh bounding box (:523-553)
  for (size_t r = 1; r < colors.size(); ++r) {
    for (int64_t i = 1; i <= nn; ++i) {
      if (node_col[i] != colors[r]) continue;
      const double* x = &nodes[3 * (i - 1)];
      bool hit = false;
      for (int d = 0; d < 3 && !hit; ++d)
        hit = (std::fabs(x[d] - xmin[d]) < 0.1 * in.delta[d]) || (std::fabs(x[d] - xmax[d]) < 0.1 * in.delta[d]);
      if (hit) { tb[r] = 1; break; }
    }
  }
  // mark kept regions with -1 (:572-593)
  for (size_t r = 0; r < colors.size(); ++r) {
    if (!tb[r]) continue;
    for (int64_t i = 1; i <= nn; ++i) if (node_col[i] == colors[r]) node_col[i] = -1;
    for (int64_t e = 1; e <= ne; ++e) if (elem_col[e] == colors[r]) elem_col[e] = -1;
  }
  // delete unconnected elements; the last element always survives (:598-613)
  {
    int64_t jj = 1, kk = 1;
    while (jj < ne) {
      if (elem_col[jj] != -1) { jj += 1; } else { jj += 1; kk += 1; }
      elem_col[kk] = elem_col[jj];
      for (int a = 0; a < nen; ++a) elems[(kk - 1) * nen + a] = elems[(jj - 1) * nen + a];
      evox[kk - 1] = evox[jj - 1];
    }
    ne = kk;
  }
  // delete unconnected nodes; node 1 and the last node always survive (:618-648)
  std::vector<int64_t> node_cref(nn + 1, 0);
  {
    int64_t jj = 1, kk = 1;
    if (node_col[jj] == -1) {
      node_col[kk] = node_col[jj];
      for (int d = 0; d < 3; ++d) nodes[3 * (kk - 1) + d] = nodes[3 * (jj - 1) + d];
      node_cref[jj] = kk;
    }
    for (;;) {
      if (node_col[jj] != -1) { node_cref[jj] = 0; node_col[jj] = 0; jj += 1; }
      else { jj += 1; kk += 1; }
      node_col[kk] = node_col[jj];
      for (int d = 0; d < 3; ++d) nodes[3 * (kk - 1) + d] = nodes[3 * (jj - 1) + d];
      node_cref[jj] = kk;
      if (jj == nn) break;
    }
    nn = kk;
  }
  for (int64_t e = 0; e < ne * nen; ++e) elems[e] = node_cref[elems[e]];
  elems.resize(ne * nen);
  evox.resize(ne);
  nodes.resize(3 * nn);
  m.ne = ne; m.nn = nn;
  m.elems.swap(elems); m.evox.swap(evox); m.nodes.swap(nodes);
  return true;
}

// ---------------------------------------------------------------------------------------
// Boundary conditions: generate_boundaries (mod_struct_preprocess.f90:490-738) with one
// mesh part, and determine_prescribed_displ (mod_write_deck.f90:22-51) for the macro order
// (8 macro nodes / 24 load cases or 20 / 60).
struct BC {
  std::vector<int64_t> ids;   // constrained node ids in node order
  std::vector<double> vals;   // (nl, 3*nb) column-major
};

void generate_boundaries(const orc_domain_in& in, const Mesh& m, BC& bc, double min_c[3], double max_c[3]) {
  double dim_c[3];
  for (int d = 0; d < 3; ++d) {
    min_c[d] = (double)(in.xa_n[d] - 1) * in.delta[d];
    max_c[d] = (double)(in.xa_n[d] + in.L[d] - 1) * in.delta[d];   // xe_n * delta
    dim_c[d] = (double)in.L[d] * in.delta[d];                       // x_D_phy
  }
  const int nm = in.macro_order == 2 ? 20 : 8, nl = 3 * nm;
  std::vector<double> uu(nm * 3 * nl);
  if (nm == 20) boundary_modes20(kEpsBC, uu.data());
  else boundary_modes(kEpsBC, uu.data());
  for (int64_t i = 0; i < m.nn; ++i) {
    const double* c = &m.nodes[3 * i];
    bool on = ((c[2] - min_c[2]) <= (dim_c[2] * kDeltaB)) || ((max_c[2] - c[2]) <= (dim_c[2] * kDeltaB)) ||
              ((c[1] - min_c[1]) <= (dim_c[1] * kDeltaB)) || ((max_c[1] - c[1]) <= (dim_c[1] * kDeltaB)) ||
              ((c[0] - min_c[0]) <= (dim_c[0] * kDeltaB)) || ((max_c[0] - c[0]) <= (dim_c[0] * kDeltaB));
    if (on) bc.ids.push_back(i + 1);
  }
  // bnode_vals(lc, 3*(b-1)+comp), column-major; each value is a left-to-right Fortran SUM
  const int64_t nb = (int64_t)bc.ids.size();
  bc.vals.assign(nl * 3 * nb, 0.0);
  for (int64_t b = 0; b < nb; ++b) {
    const double* c = &m.nodes[3 * (bc.ids[b] - 1)];
    double xi[3], N[20];
    t_geom_xi(c, min_c, max_c, xi);
    phi_nn_macro(nm, xi, N);
    for (int comp = 0; comp < 3; ++comp)
      for (int lc = 0; lc < nl; ++lc) {
        double s = 0.0;
        for (int l = 0; l < nm; ++l) s += N[l] * uu[l + nm * comp + nl * lc];
        bc.vals[lc + nl * (3 * b + comp)] = s;
      }
  }
}

// ---------------------------------------------------------------------------------------
// Assembled CSR (MatSetValues ADD_VALUES in element order, negative dof ids ignored as
// PETSc does; mod_dtc_main_subroutines.f90:516-579).
struct CSR {
  int64_t n = 0;
  std::vector<int64_t> ptr, col;
  std::vector<double> val;
  void mult(const double* x, double* y, int nrhs) const {  // y = A x, x/y [n][nrhs]
    for (int64_t i = 0; i < n; ++i) {
      double acc[60];
      for (int r = 0; r < nrhs; ++r) acc[r] = 0.0;
      for (int64_t p = ptr[i]; p < ptr[i + 1]; ++p) {
        const double a = val[p];
        const double* xr = x + col[p] * nrhs;
        for (int r = 0; r < nrhs; ++r) acc[r] += a * xr[r];
      }
      for (int r = 0; r < nrhs; ++r) y[i * nrhs + r] = acc[r];
    }
  }
};

void assemble(const orc_domain_in& in, const Mesh& m, const double* ke, CSR& A) {
  const int nen = in.nen, nd = 3 * nen;
  const int64_t ndof = 3 * m.nn;
  std::vector<std::vector<int64_t>> adj(m.nn);
  for (int64_t e = 0; e < m.ne; ++e)
    for (int a = 0; a < nen; ++a) {
      int64_t na = m.elems[e * nen + a];
      if (na <= 0) continue;
      for (int b = 0; b < nen; ++b) {
        int64_t nb = m.elems[e * nen + b];
        if (nb > 0) adj[na - 1].push_back(nb - 1);
      }
    }
  for (auto& v : adj) { std::sort(v.begin(), v.end()); v.erase(std::unique(v.begin(), v.end()), v.end()); }
  A.n = ndof;
  A.ptr.assign(ndof + 1, 0);
  for (int64_t i = 0; i < m.nn; ++i)
    for (int c = 0; c < 3; ++c) A.ptr[3 * i + c + 1] = (int64_t)adj[i].size() * 3;
  for (int64_t i = 0; i < ndof; ++i) A.ptr[i + 1] += A.ptr[i];
  A.col.resize(A.ptr[ndof]);
  A.val.assign(A.ptr[ndof], 0.0);
  for (int64_t i = 0; i < m.nn; ++i)
    for (int c = 0; c < 3; ++c) {
      int64_t p = A.ptr[3 * i + c];
      for (int64_t j : adj[i])
        for (int cj = 0; cj < 3; ++cj) A.col[p++] = 3 * j + cj;
    }
  const double escale_ref = in.E;
  for (int64_t e = 0; e < m.ne; ++e) {
    double s = 1.0;
    if (in.E_voxel) s = (double)in.E_voxel[m.evox[e]] / escale_ref;
    for (int a = 0; a < nen; ++a) {
      int64_t na = m.elems[e * nen + a];
      if (na <= 0) continue;
      for (int ci = 0; ci < 3; ++ci) {
        int64_t row = 3 * (na - 1) + ci;
        for (int b = 0; b < nen; ++b) {
          int64_t nb = m.elems[e * nen + b];
          if (nb <= 0) continue;
          for (int cj = 0; cj < 3; ++cj) {
            int64_t colv = 3 * (nb - 1) + cj;
            int64_t lo = A.ptr[row], hi = A.ptr[row + 1];
            int64_t p = std::lower_bound(A.col.begin() + lo, A.col.begin() + hi, colv) - A.col.begin();
            double kv = ke[(3 * a + ci) + nd * (3 * b + cj)];
            A.val[p] += in.E_voxel ? s * kv : kv;
          }
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------------------
// PETSc KSPSolve_CG (3.18) with PCJACOBI and KSPConvergedDefault semantics, zero initial
// guess, preconditioned 2-norm; the 24 right-hand sides are advanced side by side, each
// with exactly the arithmetic of a separate solve.
struct CGState { double beta = 0, betaold = 1, dpi = 0, dpiold = 0, dp0 = 0; int64_t its = 0; int reason = 0; };

void pcg_batch(const CSR& A, const std::vector<double>& dinv, const double* b, double* x,
               int nrhs, double rtol, int64_t max_it, int64_t* its_out, int* reason_out) {
  // Row-major passes over all columns; each column's sums run over the dofs in index
  // order, exactly as a separate solve would.  Stopped columns get alpha = 0 (x, r frozen).
  const int64_t n = A.n;
  const int R = nrhs;
  std::vector<double> r(b, b + n * R), z(n * R), p(n * R, 0.0), w(n * R);
  std::fill(x, x + n * R, 0.0);
  std::vector<CGState> st(R);
  const double abstol = 1e-50, divtol = 1e5;
  std::vector<double> s1(R), s2(R), coef(R);
  std::vector<char> active(R, 1);
  auto precond_and_dots = [&]() {   // z = D^-1 r ; s1 = z.z ; s2 = z.r
    std::fill(s1.begin(), s1.end(), 0.0);
    std::fill(s2.begin(), s2.end(), 0.0);
    for (int64_t i = 0; i < n; ++i) {
      const double d = dinv[i];
      double* zi = &z[i * R];
      const double* ri = &r[i * R];
      for (int c = 0; c < R; ++c) {
        zi[c] = d * ri[c];
        s1[c] += zi[c] * zi[c];
        s2[c] += zi[c] * ri[c];
      }
    }
  };
  precond_and_dots();
  for (int c = 0; c < R; ++c) {
    double dp = std::sqrt(s1[c]);
    st[c].dp0 = dp;
    double ttol = std::max(rtol * dp, abstol);
    if (std::isnan(dp) || std::isinf(dp)) { st[c].reason = -9; active[c] = 0; continue; }
    if (dp <= ttol) { st[c].reason = 2; active[c] = 0; continue; }
    st[c].beta = s2[c];
  }
  for (int64_t i = 0; i < max_it; ++i) {
    bool any = false;
    for (int c = 0; c < R; ++c) {
      coef[c] = 0.0;
      if (!active[c]) continue;
      st[c].its = i + 1;
      if (st[c].beta == 0.0) { st[c].reason = 3; active[c] = 0; continue; }
      if (i > 0 && st[c].beta * st[c].betaold < 0.0) { st[c].reason = -8; active[c] = 0; continue; }
      coef[c] = (i == 0) ? 0.0 : st[c].beta / st[c].betaold;
      any = true;
    }
    if (!any) break;
    for (int64_t k = 0; k < n * R; k += R)
      for (int c = 0; c < R; ++c)
        if (active[c]) p[k + c] = (i == 0) ? z[k + c] : z[k + c] + coef[c] * p[k + c];
    A.mult(p.data(), w.data(), R);
    std::fill(s1.begin(), s1.end(), 0.0);
    for (int64_t k = 0; k < n * R; k += R)
      for (int c = 0; c < R; ++c) s1[c] += p[k + c] * w[k + c];
    for (int c = 0; c < R; ++c) {
      coef[c] = 0.0;
      if (!active[c]) continue;
      st[c].dpiold = st[c].dpi;
      st[c].dpi = s1[c];
      st[c].betaold = st[c].beta;
      double sg1 = (st[c].dpi > 0) - (st[c].dpi < 0), sg0 = (st[c].dpiold > 0) - (st[c].dpiold < 0);
      if (st[c].dpi == 0.0 || (i > 0 && sg1 * sg0 < 0.0)) { st[c].reason = -8; active[c] = 0; continue; }
      coef[c] = st[c].beta / st[c].dpi;
    }
    for (int64_t k = 0; k < n * R; k += R)
      for (int c = 0; c < R; ++c) {
        x[k + c] += coef[c] * p[k + c];
        r[k + c] -= coef[c] * w[k + c];
      }
    precond_and_dots();
    bool any2 = false;
    for (int c = 0; c < R; ++c) {
      if (!active[c]) continue;
      double dp = std::sqrt(s1[c]);
      double ttol = std::max(rtol * st[c].dp0, abstol);
      if (std::isnan(dp) || std::isinf(dp)) { st[c].reason = -9; active[c] = 0; continue; }
      if (dp <= ttol) { st[c].reason = 2; active[c] = 0; continue; }
      if (dp >= divtol * st[c].dp0) { st[c].reason = -4; active[c] = 0; continue; }
      st[c].beta = s2[c];
      any2 = true;
    }
    if (!any2) break;
  }
  for (int c = 0; c < R; ++c) {
    if (active[c]) st[c].reason = -3;  // KSP_DIVERGED_ITS
    its_out[c] = st[c].its;
    reason_out[c] = st[c].reason;
  }
}

// ---------------------------------------------------------------------------------------
// LINPACK-style inverse: LU with partial pivoting (first maximal |pivot|), then the
// inverse from the factors (linpack/mod_linpack.f90:10-62, dgefa/dgedi).
bool inverse(int n, double* a) {
  std::vector<int> ipvt(n);
  for (int k = 0; k < n - 1; ++k) {
    int l = k;
    double mx = std::fabs(a[k + n * k]);
    for (int i = k + 1; i < n; ++i) if (std::fabs(a[i + n * k]) > mx) { mx = std::fabs(a[i + n * k]); l = i; }
    ipvt[k] = l;
    if (a[l + n * k] == 0.0) return false;
    if (l != k) std::swap(a[l + n * k], a[k + n * k]);
    double t = -1.0 / a[k + n * k];
    for (int i = k + 1; i < n; ++i) a[i + n * k] *= t;
    for (int j = k + 1; j < n; ++j) {
      double tj = a[l + n * j];
      if (l != k) { a[l + n * j] = a[k + n * j]; a[k + n * j] = tj; }
      for (int i = k + 1; i < n; ++i) a[i + n * j] += tj * a[i + n * k];
    }
  }
  ipvt[n - 1] = n - 1;
  if (a[(n - 1) + n * (n - 1)] == 0.0) return false;
  // inverse(U)
  for (int k = 0; k < n; ++k) {
    a[k + n * k] = 1.0 / a[k + n * k];
    double t = -a[k + n * k];
    for (int i = 0; i < k; ++i) a[i + n * k] *= t;
    for (int j = k + 1; j < n; ++j) {
      double tj = a[k + n * j];
      a[k + n * j] = 0.0;
      for (int i = 0; i <= k; ++i) a[i + n * j] += tj * a[i + n * k];
    }
  }
  // inverse(U) * inverse(L)
  std::vector<double> work(n);
  for (int kb = 0; kb < n - 1; ++kb) {
    int k = n - 2 - kb;
    for (int i = k + 1; i < n; ++i) { work[i] = a[i + n * k]; a[i + n * k] = 0.0; }
    for (int j = k + 1; j < n; ++j) {
      double t = work[j];
      for (int i = 0; i < n; ++i) a[i + n * k] += t * a[i + n * j];
    }
    int l = ipvt[k];
    if (l != k) for (int i = 0; i < n; ++i) std::swap(a[i + n * k], a[i + n * l]);
  }
  return true;
}

void matmul(int n, int m, int p, const double* a, const double* b, double* c) {  // c(n,p)=a(n,m)b(m,p)
  for (int j = 0; j < p; ++j)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int k = 0; k < m; ++k) s += a[i + n * k] * b[k + m * j];
      c[i + n * j] = s;
    }
}

// check_sym (geb-lib, absent): own definition max|A-A^T| / max|A| (0 for A = 0).
double check_sym(int n, const double* a) {
  double d = 0, s = 0;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      d = std::max(d, std::fabs(a[i + n * j] - a[j + n * i]));
      s = std::max(s, std::fabs(a[i + n * j]));
    }
  return s > 0 ? d / s : 0.0;
}

// ---------------------------------------------------------------------------------------
// Rotation search (mod_struct_calcmat.f90:533-1603)
struct Rot { double aa[9]; double BB[36]; };  // column-major

inline void rot_alg(const double n[3], double alpha, double* aa) {  // inline form :556-574
  double ca = std::cos(alpha), sa = std::sin(alpha), omc = 1.0 - ca;
  double n12 = n[0] * n[1], n13 = n[0] * n[2], n23 = n[1] * n[2];
  auto A = [&](int i, int j) -> double& { return aa[(i - 1) + 3 * (j - 1)]; };
  A(1, 1) = ca + n[0] * n[0] * omc;
  A(2, 2) = ca + n[1] * n[1] * omc;
  A(3, 3) = ca + n[2] * n[2] * omc;
  A(1, 2) = n12 * omc - n[2] * sa;
  A(2, 1) = n12 * omc + n[2] * sa;
  A(1, 3) = n13 * omc + n[1] * sa;
  A(3, 1) = n13 * omc - n[1] * sa;
  A(2, 3) = n23 * omc - n[0] * sa;
  A(3, 2) = n23 * omc + n[0] * sa;
}

inline void tra_r6(const double* aa, double* BB) {  // inline form :578-589
  auto a = [&](int i, int j) { return aa[(i - 1) + 3 * (j - 1)]; };
  double* b = BB;
  auto col = [&](int j, double v1, double v2, double v3, double v4, double v5, double v6) {
    double* c = b + 6 * (j - 1);
    c[0] = v1; c[1] = v2; c[2] = v3; c[3] = v4; c[4] = v5; c[5] = v6;
  };
  col(1, a(1, 1) * a(1, 1), a(2, 1) * a(2, 1), a(3, 1) * a(3, 1), kSq2 * a(2, 1) * a(1, 1), kSq2 * a(1, 1) * a(3, 1), kSq2 * a(2, 1) * a(3, 1));
  col(2, a(1, 2) * a(1, 2), a(2, 2) * a(2, 2), a(3, 2) * a(3, 2), kSq2 * a(2, 2) * a(1, 2), kSq2 * a(1, 2) * a(3, 2), kSq2 * a(2, 2) * a(3, 2));
  col(3, a(1, 3) * a(1, 3), a(2, 3) * a(2, 3), a(3, 3) * a(3, 3), kSq2 * a(2, 3) * a(1, 3), kSq2 * a(1, 3) * a(3, 3), kSq2 * a(2, 3) * a(3, 3));
  col(4, kSq2 * a(1, 1) * a(1, 2), kSq2 * a(2, 1) * a(2, 2), kSq2 * a(3, 1) * a(3, 2),
      a(2, 1) * a(1, 2) + a(2, 2) * a(1, 1), a(1, 1) * a(3, 2) + a(1, 2) * a(3, 1), a(2, 1) * a(3, 2) + a(2, 2) * a(3, 1));
  col(5, kSq2 * a(1, 1) * a(1, 3), kSq2 * a(2, 1) * a(2, 3), kSq2 * a(3, 1) * a(3, 3),
      a(2, 1) * a(1, 3) + a(2, 3) * a(1, 1), a(1, 1) * a(3, 3) + a(1, 3) * a(3, 1), a(2, 1) * a(3, 3) + a(2, 3) * a(3, 1));
  col(6, kSq2 * a(1, 2) * a(1, 3), kSq2 * a(2, 2) * a(2, 3), kSq2 * a(3, 2) * a(3, 3),
      a(2, 2) * a(1, 3) + a(2, 3) * a(1, 2), a(1, 2) * a(3, 3) + a(1, 3) * a(3, 2), a(2, 2) * a(3, 3) + a(2, 3) * a(3, 2));
}

// (B^T E B)(i,j) in the unrolled order of :591-761: sum over r = 6..1 of
// B(r,i) * (sum over c = 6..1 of B(c,j) E(r,c)).
inline double tbeb(const double* BB, const double* EE, int i, int j) {
  auto B = [&](int r, int c) { return BB[(r - 1) + 6 * (c - 1)]; };
  auto E = [&](int r, int c) { return EE[(r - 1) + 6 * (c - 1)]; };
  double t = 0.0;
  for (int r = 6; r >= 1; --r) {
    double s = B(6, j) * E(r, 6);
    for (int c = 5; c >= 1; --c) s = s + B(c, j) * E(r, c);
    t = (r == 6) ? B(r, i) * s : t + B(r, i) * s;
  }
  return t;
}

inline void unit_normal(double phi, double eta, double n[3]) {
  n[0] = std::cos(phi) * std::sin(eta);
  n[1] = std::sin(phi) * std::sin(eta);
  n[2] = std::cos(eta);
  double s = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  n[0] /= s; n[1] /= s; n[2] /= s;
}

// sin and cos of a candidate angle, rounded to nearest from quad precision (libquadmath).
// The reference takes them from its platform's libm; the argmin of the deep refinement
// levels is decided by their last bits, and glibc's double sin/cos differ from the nearest
// double for a fraction of a percent of these arguments, so both this oracle and the GPU
// code use the correctly rounded values (the GPU code computes them itself).
struct SinCos { double s, c; };
inline SinCos sincos_nearest(double x) {
  const __float128 q = (__float128)x;
  return {(double)sinq(q), (double)cosq(q)};
}

// criteria from the sines and cosines of (alpha, phi, eta); same expressions as rot_alg /
// unit_normal with the trigonometric values supplied
inline void criteria_sc(const double* EE, SinCos a, SinCos p, SinCos e, double* c1, double* c2) {
  double n[3] = {p.c * e.s, p.s * e.s, e.c};
  double s = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  n[0] /= s; n[1] /= s; n[2] /= s;
  double aa[9], BB[36];
  {
    double ca = a.c, sa = a.s, omc = 1.0 - ca;
    double n12 = n[0] * n[1], n13 = n[0] * n[2], n23 = n[1] * n[2];
    auto A = [&](int i, int j) -> double& { return aa[(i - 1) + 3 * (j - 1)]; };
    A(1, 1) = ca + n[0] * n[0] * omc;
    A(2, 2) = ca + n[1] * n[1] * omc;
    A(3, 3) = ca + n[2] * n[2] * omc;
    A(1, 2) = n12 * omc - n[2] * sa;
    A(2, 1) = n12 * omc + n[2] * sa;
    A(1, 3) = n13 * omc + n[1] * sa;
    A(3, 1) = n13 * omc - n[1] * sa;
    A(2, 3) = n23 * omc - n[0] * sa;
    A(3, 2) = n23 * omc + n[0] * sa;
  }
  tra_r6(aa, BB);
  double t[13];
  const int ij[12][2] = {{1, 4}, {1, 5}, {1, 6}, {2, 4}, {2, 5}, {2, 6}, {3, 4}, {3, 5}, {3, 6}, {4, 5}, {4, 6}, {5, 6}};
  for (int k = 0; k < 12; ++k) t[k + 1] = tbeb(BB, EE, ij[k][0], ij[k][1]);
  *c1 = t[2] * t[2] + t[3] * t[3] + t[5] * t[5] + t[6] * t[6] + t[8] * t[8] + t[9] * t[9] + t[10] * t[10] + t[11] * t[11];
  *c2 = t[1] * t[1] + t[2] * t[2] + t[3] * t[3] + t[4] * t[4] + t[5] * t[5] + t[6] * t[6] + t[7] * t[7] + t[8] * t[8] +
        t[9] * t[9] + t[10] * t[10] + t[11] * t[11] + t[12] * t[12];
}

// One criterion's sweep + x10 refinement (mod_struct_calcmat.f90:762-1012 / :1206-1460);
// returns angles (integers in units of 10^-jj deg) and jj.  MINLOC picks the first minimum
// in column-major order (alpha fastest).  The angle of index i at a level is i * div with
// div = (pi/180) * 0.1^jj formed by repeated multiplication, as the reference forms it.
void search_one(const double* EE, int which, int64_t ang_out[3], int* jj_out, double* crit_out) {
  SinCos deg[181];
  for (int k = 0; k <= 180; ++k) deg[k] = sincos_nearest((double)k * kPiDiv180);
  double best = INFINITY;
  int64_t ba = 0, bp = 0, be = 0;
  for (int ie = 0; ie <= 90; ++ie)
    for (int ip = 0; ip <= 180; ++ip)
      for (int ia = 0; ia <= 180; ++ia) {
        double c1, c2;
        criteria_sc(EE, deg[ia], deg[ip], deg[ie], &c1, &c2);
        double c = which == 1 ? c1 : c2;
        if (c < best) { best = c; ba = ia; bp = ip; be = ie; }
      }
  double crit_min[17];
  for (int i = 0; i < 17; ++i) crit_min[i] = 0.0;
  crit_min[0] = best;
  int jj = 1;
  double div = kPiDiv180;
  int64_t ca = ba, cp = bp, ce = be;
  for (;;) {
    int64_t s[3] = {(ca - 1) * 10, (cp - 1) * 10, (ce - 1) * 10};
    int64_t e[3] = {(ca + 1) * 10, (cp + 1) * 10, (ce + 1) * 10};
    div = div * 0.1;
    SinCos tab[3][21];
    for (int d = 0; d < 3; ++d)
      for (int64_t i = s[d]; i <= e[d]; ++i) tab[d][i - s[d]] = sincos_nearest((double)i * div);
    double wbest = INFINITY;
    int64_t na = 0, np = 0, nE = 0;
    for (int64_t ie = s[2]; ie <= e[2]; ++ie)
      for (int64_t ip = s[1]; ip <= e[1]; ++ip)
        for (int64_t ia = s[0]; ia <= e[0]; ++ia) {
          double c1, c2;
          criteria_sc(EE, tab[0][ia - s[0]], tab[1][ip - s[1]], tab[2][ie - s[2]], &c1, &c2);
          double c = which == 1 ? c1 : c2;
          if (c < wbest) { wbest = c; na = ia; np = ip; nE = ie; }
        }
    crit_min[jj] = wbest;
    ca = na; cp = np; ce = nE;
    if ((std::fabs(crit_min[jj - 1] - crit_min[jj]) < kNumZero) || (jj >= 16)) break;
    jj += 1;
  }
  ang_out[0] = ca; ang_out[1] = cp; ang_out[2] = ce;
  *jj_out = jj;
  *crit_out = crit_min[jj];
}

// axis-permutation fix-up so that E11 <= E22 <= E33 (:1066-1134 / :1510-1576)
void permutation_fixup(const double* EE, double n[3], double* alpha, double* aa) {
  auto E = [&](int i) { return EE[(i - 1) + 6 * (i - 1)]; };
  auto rot_mul = [&](int colidx) {
    double nn[3] = {aa[0 + 3 * colidx], aa[1 + 3 * colidx], aa[2 + 3 * colidx]};
    double R[9], out[9];
    rot_alg(nn, kPi / 2, R);
    matmul(3, 3, 3, R, aa, out);
    std::memcpy(aa, out, sizeof(out));
    n[0] = nn[0]; n[1] = nn[1]; n[2] = nn[2];
    *alpha = kPi / 2;
  };
  double e1 = E(1), e2 = E(2), e3 = E(3);
  if (e1 < e2 && e1 < e3 && e2 < e3) {
  } else if (e1 < e2 && e1 < e3 && e2 > e3) {
    rot_mul(0);
  } else if (e1 < e2 && e1 > e3 && e2 > e3) {
    rot_mul(1); rot_mul(0);
  } else if (e1 > e2 && e1 < e3 && e2 < e3) {
    rot_mul(2);
  } else if (e1 > e2 && e1 > e3 && e2 < e3) {
    rot_mul(2); rot_mul(0);
  } else if (e1 > e2 && e1 > e3 && e2 > e3) {
    rot_mul(1);
  }
}

void rotate_tensor(const double* aa, const double* EEo, double* EEr) {
  double BB[36], BT[36], tmp[36];
  tra_r6(aa, BB);
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) BT[i + 6 * j] = BB[j + 6 * i];
  matmul(6, 6, 6, BT, EEo, tmp);
  matmul(6, 6, 6, tmp, BB, EEr);
}

void rotation_search(const double* EE, orc_domain_out* out) {
  for (int which = 1; which <= 2; ++which) {
    int64_t ang[3]; int jj; double crit;
    search_one(EE, which, ang, &jj, &crit);
    double scale = kPi / (180.0 * (std::pow(10.0, jj) - 1));   // quirk: 10**jj - 1 (:1017)
    double alpha = (double)ang[0] * scale, phi = (double)ang[1] * scale, eta = (double)ang[2] * scale;
    double n[3], aa[9], EEr[36];
    unit_normal(phi, eta, n);
    rot_alg(n, alpha, aa);
    rotate_tensor(aa, EE, EEr);
    double n_out[3] = {n[0], n[1], n[2]}, alpha_out = alpha;   // CR1 writes angle/vector before the fix-up
    permutation_fixup(EEr, n, &alpha, aa);
    rotate_tensor(aa, EE, EEr);
    if (which == 1) {
      out->cr1_angle = alpha_out; std::memcpy(out->cr1_n, n_out, sizeof(n_out));
      std::memcpy(out->cr1_aa, aa, sizeof(aa)); std::memcpy(out->cr1_ee, EEr, sizeof(EEr));
      out->cr1_crit = crit; out->cr1_iters = jj;
      std::memcpy(out->cr1_ang, ang, sizeof(ang));
    } else {                                                     // CR2 writes them after it (:1583-1597)
      out->cr2_angle = alpha; std::memcpy(out->cr2_n, n, sizeof(n));
      std::memcpy(out->cr2_aa, aa, sizeof(aa)); std::memcpy(out->cr2_ee, EEr, sizeof(EEr));
      out->cr2_crit = crit; out->cr2_iters = jj;
      std::memcpy(out->cr2_ang, ang, sizeof(ang));
    }
  }
}

// ---------------------------------------------------------------------------------------
int validate(const orc_domain_in* in) {
  if (!in || !in->phi) return ORC_BAD_INPUT;
  if (in->nen != 8 && in->nen != 20) return ORC_BAD_INPUT;
  for (int d = 0; d < 3; ++d) if (in->L[d] < 1 || in->delta[d] <= 0) return ORC_BAD_INPUT;
  return ORC_OK;
}

int run_domain(const orc_domain_in* in, orc_domain_out* out, bool solve) {
  int st = validate(in);
  if (st) { out->status = st; return st; }
  out->status = ORC_OK;
  out->ne = out->nn = out->nb = 0;
  const int nm = in->macro_order == 2 ? 20 : 8, nl = 3 * nm;   // macro nodes, load cases
  for (int i = 0; i < 60; ++i) out->iters[i] = 0;
  Mesh m;
  if (!gen_quadmesh(*in, m)) { out->status = ORC_EMPTY; return ORC_EMPTY; }
  out->ne = m.ne; out->nn = m.nn;
  if (m.nn == 0 || m.ne == 0) { out->status = ORC_NO_STRUCTURE; return out->status; }
  BC bc;
  double min_c[3], max_c[3];
  generate_boundaries(*in, m, bc, min_c, max_c);
  const int64_t nb = (int64_t)bc.ids.size();
  out->nb = nb;
  if (out->elems && out->cap_elems >= m.ne) std::memcpy(out->elems, m.elems.data(), sizeof(int64_t) * m.elems.size());
  if (out->elem_voxel && out->cap_elems >= m.ne) std::memcpy(out->elem_voxel, m.evox.data(), sizeof(int64_t) * m.ne);
  if (out->nodes && out->cap_nodes >= m.nn) std::memcpy(out->nodes, m.nodes.data(), sizeof(double) * m.nodes.size());
  if (out->bnode_ids && out->cap_nodes >= m.nn) std::memcpy(out->bnode_ids, bc.ids.data(), sizeof(int64_t) * nb);
  if (out->bnode_vals && out->cap_nodes >= m.nn) std::memcpy(out->bnode_vals, bc.vals.data(), sizeof(double) * bc.vals.size());
  if (m.nn < 6) { out->status = ORC_FEW_NODES; return out->status; }  // :471-473 (node-count leaf)
  if (!solve) return ORC_OK;

  const int nen = in->nen, nd = 3 * nen;
  std::vector<double> ke(nd * nd);
  element_stiffness(nen, in->E, in->phdsize[0] * in->delta[0], in->nu, ke.data());  // a = phdsize(1)*delta(1)
  CSR A;
  assemble(*in, m, ke.data(), A);
  const CSR& Aorg = A;  // AA_org keeps the assembled values
  const int64_t n = A.n;
  // bc dofs and values per load case
  std::vector<int64_t> gdof(3 * nb);
  for (int64_t b = 0; b < nb; ++b) for (int c = 0; c < 3; ++c) gdof[3 * b + c] = 3 * (bc.ids[b] - 1) + c;
  std::vector<double> XX(n * nl, 0.0), F(n * nl, 0.0);
  for (int64_t k = 0; k < 3 * nb; ++k)
    for (int lc = 0; lc < nl; ++lc) XX[gdof[k] * nl + lc] = -bc.vals[lc + nl * k];
  Aorg.mult(XX.data(), F.data(), nl);                       // F_lc = A (-u_c)  (:674-933)
  for (int64_t k = 0; k < 3 * nb; ++k) for (int lc = 0; lc < nl; ++lc) F[gdof[k] * nl + lc] = 0.0;
  // MatZeroRowsColumns(AA, bc, diag = 0) (:945-951); b is already consistent for every load case
  CSR Az = A;
  std::vector<char> isbc(n, 0);
  for (int64_t k = 0; k < 3 * nb; ++k) isbc[gdof[k]] = 1;
  for (int64_t i = 0; i < n; ++i)
    for (int64_t p = Az.ptr[i]; p < Az.ptr[i + 1]; ++p)
      if (isbc[i] || isbc[Az.col[p]]) Az.val[p] = 0.0;
  // PCJACOBI: zero diagonal entries are replaced by one
  std::vector<double> dinv(n, 1.0);
  for (int64_t i = 0; i < n; ++i) {
    double d = 0.0;
    for (int64_t p = Az.ptr[i]; p < Az.ptr[i + 1]; ++p) if (Az.col[p] == i) d = Az.val[p];
    dinv[i] = 1.0 / (d == 0.0 ? 1.0 : d);
  }
  std::vector<double> X(n * nl);
  int reasons[60];
  pcg_batch(Az, dinv, F.data(), X.data(), nl, in->rtol, in->max_it, out->iters, reasons);
  for (int lc = 0; lc < nl; ++lc) {
    if (reasons[lc] == -3 && out->status == ORC_OK) out->status = ORC_MAX_IT;
    if (reasons[lc] == -8 && out->status == ORC_OK) out->status = ORC_BREAKDOWN;
    if ((reasons[lc] == -9 || reasons[lc] == -4) && out->status == ORC_OK) out->status = ORC_NONFINITE;
  }
  // reactions: XX[bc] = u_c ; F = AA_org XX  (:1092-1123)
  for (int64_t k = 0; k < 3 * nb; ++k) for (int lc = 0; lc < nl; ++lc) X[gdof[k] * nl + lc] = bc.vals[lc + nl * k];
  Aorg.mult(X.data(), F.data(), nl);
  if (out->displ && out->cap_nodes >= m.nn)
    for (int lc = 0; lc < nl; ++lc) for (int64_t i = 0; i < n; ++i) out->displ[lc * n + i] = X[i * nl + lc];
  if (out->force && out->cap_nodes >= m.nn)
    for (int lc = 0; lc < nl; ++lc) for (int64_t i = 0; i < n; ++i) out->force[lc * n + i] = F[i * nl + lc];

  // calc_effective_material_parameters (mod_struct_calcmat.f90:23-1673)
  std::vector<double> vv(nl * nl);
  if (nm == 20) loadcase_matrix_quad(in->rve_strain, vv.data());
  else loadcase_matrix(in->rve_strain, vv.data());
  inverse(nl, vv.data());
  double* ff = out->ff;   // ff(nl, nl), column-major
  std::fill(ff, ff + nl * nl, 0.0);
  for (int lc = 0; lc < nl; ++lc)
    for (int64_t j = 0; j < m.nn; ++j) {
      double xi[3], N[20];
      t_geom_xi(&m.nodes[3 * j], min_c, max_c, xi);
      phi_nn_macro(nm, xi, N);
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < nm; ++l) ff[(k * nm + l) + nl * lc] = ff[(k * nm + l) + nl * lc] + F[(3 * j + k) * nl + lc] * N[l];
    }
  matmul(nl, nl, nl, ff, vv.data(), out->kmacro);
  out->sym_k = check_sym(nl, out->kmacro);
  double xdp[3] = {(double)in->L[0] * in->delta[0], (double)in->L[1] * in->delta[1], (double)in->L[2] * in->delta[2]};
  double fv[36];
  auto f = [&](int r, int c) { return ff[(r - 1) + nl * (c - 1)]; };
  if (nm == 20) for (int ii = 1; ii <= 6; ++ii) {   // :368-401, the 8 nodes of each face
    fv[0 + 6 * (ii - 1)] = (f(2, ii) + f(3, ii) + f(6, ii) + f(7, ii) + f(10, ii) + f(14, ii) + f(18, ii) + f(19, ii)) /
                           (xdp[1] * xdp[2]);
    fv[1 + 6 * (ii - 1)] = (f(23, ii) + f(24, ii) + f(27, ii) + f(28, ii) + f(31, ii) + f(35, ii) + f(39, ii) + f(40, ii)) /
                           (xdp[0] * xdp[2]);
    fv[2 + 6 * (ii - 1)] = (f(45, ii) + f(46, ii) + f(47, ii) + f(48, ii) + f(53, ii) + f(54, ii) + f(55, ii) + f(56, ii)) /
                           (xdp[0] * xdp[1]);
    fv[3 + 6 * (ii - 1)] =
        0.5 * ((f(3, ii) + f(4, ii) + f(7, ii) + f(8, ii) + f(11, ii) + f(15, ii) + f(19, ii) + f(20, ii)) / (xdp[0] * xdp[2]) +
               (f(22, ii) + f(23, ii) + f(26, ii) + f(27, ii) + f(30, ii) + f(34, ii) + f(38, ii) + f(39, ii)) / (xdp[1] * xdp[2]));
    fv[4 + 6 * (ii - 1)] =
        0.5 * ((f(5, ii) + f(6, ii) + f(7, ii) + f(8, ii) + f(13, ii) + f(14, ii) + f(15, ii) + f(16, ii)) / (xdp[0] * xdp[1]) +
               (f(42, ii) + f(43, ii) + f(46, ii) + f(47, ii) + f(50, ii) + f(54, ii) + f(58, ii) + f(59, ii)) / (xdp[1] * xdp[2]));
    fv[5 + 6 * (ii - 1)] =
        0.5 * ((f(25, ii) + f(26, ii) + f(27, ii) + f(28, ii) + f(33, ii) + f(34, ii) + f(35, ii) + f(36, ii)) / (xdp[0] * xdp[1]) +
               (f(43, ii) + f(44, ii) + f(47, ii) + f(48, ii) + f(51, ii) + f(55, ii) + f(59, ii) + f(60, ii)) / (xdp[0] * xdp[2]));
  }
  else for (int ii = 1; ii <= 6; ++ii) {   // :345-359
    fv[0 + 6 * (ii - 1)] = (f(2, ii) + f(3, ii) + f(6, ii) + f(7, ii)) / (xdp[1] * xdp[2]);
    fv[1 + 6 * (ii - 1)] = (f(11, ii) + f(12, ii) + f(15, ii) + f(16, ii)) / (xdp[0] * xdp[2]);
    fv[2 + 6 * (ii - 1)] = (f(21, ii) + f(22, ii) + f(23, ii) + f(24, ii)) / (xdp[0] * xdp[1]);
    fv[3 + 6 * (ii - 1)] = 0.5 * ((f(3, ii) + f(4, ii) + f(7, ii) + f(8, ii)) / (xdp[0] * xdp[2]) +
                                  (f(10, ii) + f(11, ii) + f(14, ii) + f(15, ii)) / (xdp[1] * xdp[2]));
    fv[4 + 6 * (ii - 1)] = 0.5 * ((f(5, ii) + f(6, ii) + f(7, ii) + f(8, ii)) / (xdp[0] * xdp[1]) +
                                  (f(18, ii) + f(19, ii) + f(22, ii) + f(23, ii)) / (xdp[1] * xdp[2]));
    fv[5 + 6 * (ii - 1)] = 0.5 * ((f(13, ii) + f(14, ii) + f(15, ii) + f(16, ii)) / (xdp[0] * xdp[1]) +
                                  (f(19, ii) + f(20, ii) + f(23, ii) + f(24, ii)) / (xdp[0] * xdp[2]));
  }
  double meps[36] = {0};                                     // :434-439
  meps[0 + 6 * 0] = 1e6; meps[1 + 6 * 1] = 1e6; meps[2 + 6 * 2] = 1e6;
  meps[3 + 6 * 3] = -1e6; meps[4 + 6 * 4] = -1e6; meps[5 + 6 * 5] = 1e6;
  matmul(6, 6, 6, fv, meps, out->c);
  out->sym_c = check_sym(6, out->c);
  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) out->ee[i + 6 * j] = (out->c[i + 6 * j] + out->c[j + 6 * i]) / 2.0;
  out->sym_ee = check_sym(6, out->ee);
  if (in->rotation) rotation_search(out->ee, out);
  out->density = (double)m.ne / ((double)in->L[0] * (double)in->L[1] * (double)in->L[2]);  // :1642-1651
  return out->status;
}

}  // namespace

extern "C" {

int orc_solve_domain(const orc_domain_in* in, orc_domain_out* out) { return run_domain(in, out, true); }
int orc_mesh_domain(const orc_domain_in* in, orc_domain_out* out) { return run_domain(in, out, false); }

int orc_solve_batch(const orc_domain_in* in, orc_domain_out* out, int64_t n, int32_t nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int64_t i = 0; i < n; ++i) run_domain(&in[i], &out[i], true);
  return 0;
}

int orc_element_stiffness(int32_t nen, double E, double a, double nu, double* ke) {
  if (nen != 8 && nen != 20) return ORC_BAD_INPUT;
  element_stiffness(nen, E, a, nu, ke);
  return 0;
}

void orc_boundary_modes(double eps, double* uu) { boundary_modes(eps, uu); }
void orc_loadcase_matrix(double eps, double* vv) { loadcase_matrix(eps, vv); }
void orc_boundary_modes20(double eps, double* uu) { boundary_modes20(eps, uu); }
void orc_loadcase_matrix_quad(double eps, double* vv) { loadcase_matrix_quad(eps, vv); }
void orc_rotation_search(const double* ee, orc_domain_out* out) { rotation_search(ee, out); }

}  // extern "C"
