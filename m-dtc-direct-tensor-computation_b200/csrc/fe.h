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

// Homogenisation from the domain forces ff (mod_struct_calcmat.f90:216-500):
// K_macro = ff * vv^-1, fv from the face sums, C = fv * meps, EE = (C + C^T)/2.
void homogenise(const double ff[576], const int64_t L[3], const double delta[3], double rve_strain,
                dtc_domain_out* out);

// Domain forces from the energy products M(a,b) = u_a^T K u_b of the 24 load-case solutions:
// ff(r, lc) = sum_a vvbc^-1(a, r) M(a, lc), vvbc the load-case matrix of the boundary modes
// actually prescribed (eps = 1e-6, mod_write_deck.f90:61).  Equal to the reaction projection
// (mod_struct_calcmat.f90:254-280) at the exact solution.
void energy_to_ff(const double gram[576], double ff[576]);

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
