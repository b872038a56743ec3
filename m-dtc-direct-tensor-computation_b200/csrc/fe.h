// fe.h -- host-side finite-element and homogenisation helpers of the library (FP64).
#pragma once
#include <cstdint>

#include "../../include/dtc.h"

namespace dtc {

// Voxel element stiffness for unit modulus and unit edge, Poisson ratio nu, node order of
// the mesher (HEX08: mod_gen_quadmesh.f90:298-306; HEX20 ring order: :244-265).
// Column-major (3*nen)^2.  The reference's Ke (mod_linfe.f90:161-776, 890-4509) equals
// this times E * a with a = phdsize(1)*delta(1).
void voxel_stiffness(int nen, double nu, double* khat);

// Trilinear macro shape functions N_1..N_8 (mod_linfe.f90:51-66) at xi in [-1,1]^3 and
// the geometry -> xi map (mod_linfe.f90:77-84).
void macro_shape8(const double xi[3], double N[8]);
void geom_to_xi(const double x[3], const double lo[3], const double hi[3], double xi[3]);

// Prescribed macro displacement modes uu(8,3,24) (mod_write_deck.f90:63-116), column-major.
void macro_modes(double eps, double* uu);

// Boundary value of load case lc, component c at a point with shape values N.
double boundary_value(const double* uu, const double N[8], int c, int lc);

// The macro element: order 1 = 8-node trilinear brick with 24 load cases, order 2 = 20-node
// serendipity brick with 60 load cases ('Element order on macro scale',
// f-src/mod_dtc_main_subroutines.f90:498-508).
inline int macro_nodes(int order) { return order == 2 ? 20 : 8; }
inline int macro_loadcases(int order) { return order == 2 ? 60 : 24; }

// Quadratic macro shape functions N_1..N_20 in ANSYS node order (phi_NN_hexe20,
// mod_linfe.f90:827-888) and the boundary modes uu(20,3,60) of init_displ_hexe20
// (mod_write_deck.f90:118-279), column-major.
void macro_shape20(const double xi[3], double N[20]);
void macro_modes20(double eps, double* uu);

// Either order: N (8 or 20 values), uu(nm,3,nl), and the value of load case lc, component c.
void macro_shape(int order, const double xi[3], double* N);
void macro_modes_of_order(int order, double eps, double* uu);
double boundary_value_n(int nm, const double* uu, const double* N, int c, int lc);

// Load-case matrix vv(nl,nl) for eps = e (init_loadcase_el_order_lin / _quad,
// mod_struct_calcmat.f90:1684-2028): the boundary-mode table flattened component-major.  For
// order 2 this is the quadratic table of the reference with its typing defects repaired (a row
// labelled 59 that belongs at 49, 22 entries written without the factor e, one surplus
// value in row 54); every other entry of that table is reproduced exactly.
void loadcase_matrix(int order, double e, double* vv);

// Homogenisation from the domain forces ff (nl x nl, mod_struct_calcmat.f90:216-500):
// K_macro = ff * vv^-1, fv from the face sums (:345-359 order 1, :368-401 order 2),
// C = fv * meps, EE = (C + C^T)/2.  Order 2 writes ff and K_macro to out->macro2.
void homogenise(int order, const double* ff, const int64_t L[3], const double delta[3], double rve_strain,
                dtc_domain_out* out);

// Domain forces from the energy products M(a,b) = u_a^T K u_b of the nl load-case solutions:
// ff(r, lc) = sum_a vvbc^-1(a, r) M(a, lc), vvbc the load-case matrix of the boundary modes
// actually prescribed (eps = 1e-6, mod_write_deck.f90:61).  Equal to the reaction projection
// (mod_struct_calcmat.f90:254-280) at the exact solution.  gram and ff are nl x nl.
void energy_to_ff(int order, const double* gram, double* ff);

// Rotation search results -> output record (mod_struct_calcmat.f90:1014-1137, 1462-1603):
// ang = argmin indices in units of 10^-jj degree, jj = refinement iterations.
void finish_rotation(const double ee[36], int which, const int64_t ang[3], int jj, double crit,
                     dtc_domain_out* out);

// Symmetry deviation max|A - A^T| / max|A| (geb-lib check_sym is absent; own definition).
double symmetry_deviation(int n, const double* a);

// Cosines/sines of k degrees, k = 0..180, as the reference evaluates them
// (Real(k) * pi_div_180, mod_struct_calcmat.f90:546-548).
void degree_tables(double* c, double* s);

}  // namespace dtc
