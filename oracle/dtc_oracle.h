/*
 * dtc_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of the reference's per-domain homogenisation path, used as the
 * checker by tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py.
 * Nothing in the product library links or calls this code.
 *
 * Parity status: the reference (Fortran 90 + MPI + PETSc 3.18.1, geb-lib submodule
 * missing) cannot be compiled anywhere this project runs, and it ships no numeric
 * result files.  The oracle is pinned against the golden tables parsed from the
 * reference's source (tests/golden/: element stiffness tables, boundary-mode and
 * load-case tables) and against analytic known answers (isotropic solid cube);
 * the PETSc CG/Jacobi semantics it restates are cross-checked with scipy.  Beyond
 * those pins the end-to-end numbers are "parity unpinned".
 *
 * Arrays follow the reference's Fortran conventions: matrices are column-major
 * (element (i,j), 1-based, at [(i-1) + n*(j-1)]), node ids are 1-based, elements
 * list their nodes in the mesher's local order.
 */
#ifndef DTC_ORACLE_H
#define DTC_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORC_OK = 0,
  ORC_EMPTY = 1,          /* max(phi) < llimit: no mesh (mod_gen_quadmesh.f90:142-164) */
  ORC_NO_STRUCTURE = 2,   /* no nodes/elements (mod_struct_preprocess.f90:358-361) */
  ORC_FEW_NODES = 3,      /* "< 6" test on the node-count leaf (mod_struct_preprocess.f90:471-473) */
  ORC_MAX_IT = 4,         /* some load case hit max_it */
  ORC_BREAKDOWN = 5,      /* p'Ap <= 0 in CG (PETSc KSP_DIVERGED_INDEFINITE_MAT) */
  ORC_NONFINITE = 6,
  ORC_BAD_INPUT = 100
};

typedef struct {
  int64_t L[3];          /* x_D: voxels per domain edge */
  int64_t xa_n[3];       /* 1-based index of the domain's first voxel in the volume */
  int64_t llimit;        /* BINARIZE_LO */
  int32_t nen;           /* micro element: 8 (HEX08) or 20 (HEX20) */
  int32_t rotation;      /* run the CR1/CR2 rotation search */
  double delta[3];       /* voxel edge (mm) */
  double phdsize[3];     /* SIZE_DOMAIN (mm), enters the Ke factor a = phdsize(1)*delta(1) */
  double E;              /* YOUNG_MODULUS (MPa) */
  double nu;             /* POISSON_RATIO */
  double rve_strain;     /* RVE_STRAIN, the eps of the load-case matrix vv */
  double rtol;           /* KSP relative tolerance on the preconditioned residual */
  int64_t max_it;
  const int32_t* phi;    /* L0*L1*L2 gray values, x fastest */
  const float* E_voxel;  /* optional per-voxel modulus (extension); NULL -> E everywhere */
  int32_t macro_order;   /* 'Element order on macro scale': 1 (or 0) -> 8 macro nodes, nl = 24
                            load cases; 2 -> 20 macro nodes, nl = 60 */
  int32_t pad_;
} orc_domain_in;

typedef struct {
  int32_t status;
  int64_t ne, nn, nb;              /* elements, nodes, constrained nodes */
  int64_t iters[60];               /* per load case (first nl used) */
  double ff[3600];                 /* "Domain forces" ff(nl,nl), column-major with leading dimension nl */
  double kmacro[3600];             /* "Effective numerical stiffness" ff*vv^-1, nl x nl */
  double sym_k;
  double c[36];                    /* "Effective stiffness" fv*meps */
  double sym_c;
  double ee[36];                   /* "Averaged Effective stiffness" (C+C^T)/2 */
  double sym_ee;
  double cr1_angle, cr1_n[3], cr1_aa[9], cr1_ee[36], cr1_crit;
  double cr2_angle, cr2_n[3], cr2_aa[9], cr2_ee[36], cr2_crit;
  int32_t cr1_iters, cr2_iters;
  double density;
  /* optional, caller-allocated (NULL to skip) */
  int64_t cap_elems, cap_nodes;    /* capacities of the arrays below (elements, nodes) */
  int64_t* elems;                  /* nen*ne node ids (1-based; 0 = dropped by the mesher) */
  int64_t* elem_voxel;             /* ne: 0-based voxel index x+L0*(y+L1*z) of each element */
  double* nodes;                   /* 3*nn coordinates */
  int64_t* bnode_ids;              /* nb constrained node ids, in node order */
  double* bnode_vals;              /* nl x (3*nb) prescribed values, column-major like bnode_vals(nl,3nb) */
  double* displ;                   /* nl x 3nn solutions incl. BC values (lc-major) */
  double* force;                   /* nl x 3nn reaction forces AA_org*u (lc-major) */
  int64_t cr1_ang[3], cr2_ang[3];  /* argmin indices (alpha, phi, eta) in units of 10^-jj degree */
} orc_domain_out;

/* Full path for one domain: mesh -> BC -> assembly -> nl CG solves -> reactions ->
 * ff -> K_macro -> C -> EE -> rotation search. */
int orc_solve_domain(const orc_domain_in* in, orc_domain_out* out);

/* Mesh + boundary conditions only (solve skipped). */
int orc_mesh_domain(const orc_domain_in* in, orc_domain_out* out);

/* Many domains, one per OpenMP thread (the reference's domain-level MPI parallelism). */
int orc_solve_batch(const orc_domain_in* in, orc_domain_out* out, int64_t n, int32_t nthreads);

/* Element stiffness of a cube of edge a (the reference's a = phdsize*delta), modulus E,
 * Poisson nu, by Gauss quadrature; nen = 8 -> 24x24, nen = 20 -> 60x60, column-major. */
int orc_element_stiffness(int32_t nen, double E, double a, double nu, double* ke);

/* Boundary-mode table uu(8,3,24) (column-major) for eps, and vv(24,24) for eps. */
void orc_boundary_modes(double eps, double* uu);
void orc_loadcase_matrix(double eps, double* vv);

/* Macro order 2: uu(20,3,60) of init_displ_hexe20 and the repaired quadratic load-case
 * matrix vv(60,60) (init_loadcase_el_order_quad; see loadcase_matrix_quad). */
void orc_boundary_modes20(double eps, double* uu);
void orc_loadcase_matrix_quad(double eps, double* vv);

/* Rotation search alone, on a symmetric 6x6 tensor ee (column-major); fills the cr1_* and
 * cr2_* fields of out. */
void orc_rotation_search(const double* ee, orc_domain_out* out);

#ifdef __cplusplus
}
#endif
#endif
