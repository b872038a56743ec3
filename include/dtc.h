/*
 * dtc.h -- C ABI of the B200 direct-tensor-computation solver.
 *
 * Drop-in for the per-domain solve of the reference's exec_single_domain
 * (f-src/mod_dtc_main_subroutines.f90:52-1337): the block from MatCreate (:426) to
 * calc_effective_material_parameters (:1257), together with the meshing and boundary
 * generation it calls (f-src/mod_struct_preprocess.f90:23-738,
 * f-src/mod_gen_quadmesh.f90:22-679, f-src/mod_write_deck.f90:22-279) and the
 * homogenisation + rotation search (f-src/mod_struct_calcmat.f90:23-1673).
 * The MPI domain loop of the driver (f-src_main/struct_process.f90:960-1070,1240-1395)
 * becomes one call with many domains.
 *
 * Plain C types only: int64_t / double / pointers.  All arrays are caller-owned host
 * memory.  Matrices are column-major with the reference's Fortran layout (entry (i,j),
 * 1-based, at [(i-1) + n*(j-1)]), i.e. exactly the order of the reference's result leaves
 * (reshape(ff,[no_lc*no_lc]) etc., f-src/mod_struct_calcmat.f90:289-1664).
 * Functions return dtc_status; per-domain outcomes are in dtc_domain_out.status.
 * Nothing aborts the process and no device code traps.
 *
 * Threading: a handle is used by one host thread at a time; distinct handles are
 * independent.  The library owns all device memory it allocates inside a handle.
 */
#ifndef DTC_H
#define DTC_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DTC_ABI_VERSION 2

typedef enum dtc_status {
  DTC_OK = 0,
  DTC_ERR_INVALID_ARGUMENT = 1, /* a pointer, size or parameter failed validation */
  DTC_ERR_CUDA = 2,             /* a CUDA runtime call failed; see dtc_last_error */
  DTC_ERR_OUT_OF_MEMORY = 3,    /* device or host allocation failed */
  DTC_ERR_NO_DEVICE = 4,        /* no usable CUDA device */
  DTC_ERR_ABI_MISMATCH = 5,     /* dtc_options.abi_version != DTC_ABI_VERSION */
  DTC_ERR_INTERNAL = 6
} dtc_status;

/* Per-domain status, same meaning as the reference's skip paths. */
enum {
  DTC_DOMAIN_OK = 0,
  DTC_DOMAIN_EMPTY = 1,        /* max(phi) < llimit: no mesh (mod_gen_quadmesh.f90:142-164) */
  DTC_DOMAIN_NO_STRUCTURE = 2, /* no nodes or elements (mod_struct_preprocess.f90:358-361) */
  DTC_DOMAIN_FEW_NODES = 3,    /* the "< 6" test on the node-count leaf (mod_struct_preprocess.f90:471-473) */
  DTC_DOMAIN_MAX_IT = 4,       /* a load case reached max_it (KSP_DIVERGED_ITS) */
  DTC_DOMAIN_BREAKDOWN = 5,    /* p'Ap <= 0 or an indefinite preconditioner in CG */
  DTC_DOMAIN_NONFINITE = 6     /* NaN/Inf residual or divergence (KSP_DIVERGED_NANORINF/DTOL) */
};

enum { DTC_HEX08 = 8, DTC_HEX20 = 20 };

enum {
  DTC_PREC_FP64 = 0,  /* plain FP64 Jacobi-PCG, PETSc KSPCG semantics per load case */
  DTC_PREC_MIXED = 1  /* FP32 Jacobi-PCG inner solves inside FP64 iterative refinement */
};

typedef struct dtc_options {
  int32_t abi_version;     /* must be DTC_ABI_VERSION */
  int32_t precision;       /* DTC_PREC_* */
  double rtol;             /* relative tolerance on ||D^-1 r|| / ||D^-1 b|| per load case;
                              the reference's PETSc option -ksp_rtol (f-src/mod_parameters.f90:31) */
  int64_t max_it;          /* CG iteration cap per load case (-ksp_max_it, :32); for the mixed
                              path the cap on the summed inner iterations */
  double inner_rtol;       /* mixed path: reduction asked of each FP32 inner solve
                              (0 -> max(0.3 rtol, 1e-7)) */
  int32_t max_refine;      /* mixed path: cap on FP64 refinement steps (0 -> 12) */
  int32_t rotation_search; /* 1: run the CR1/CR2 rotation search (mod_struct_calcmat.f90:533-1603) */
  int32_t device;          /* CUDA device ordinal */
  int32_t host_threads;    /* threads for the host phases: meshing, packing, multigrid
                              build (0 -> the CPUs of the process affinity mask) */
  int32_t keep_displacements; /* 1: keep the converged displacements on the device for
                                 dtc_energy_grad (the adjoint); 0: release them */
  int32_t profile_kernels; /* 1: time every solver kernel with CUDA events on its stream
                              (dtc_get_kernel_stats); adds event records, off for production */
  int32_t mixed_matvec;    /* stiffness contraction of the FP32 inner solve: 0 = SIMT FP32,
                              1 = tcgen05 tensor cores (3xTF32 split, FP32-level accuracy),
                              2 = autotuned: multigrid solves time both kernels of the fine-level
                              operator on the batch's own tiles and keep the faster; for the HEX08
                              SIMT sweeps also the register budget (6 or 8 CTAs per SM) of each of
                              the residual, post-smoothing and CG-application sweeps, and for
                              every HEX08 solve that of the FP64 sweep (4 or 6 CTAs per SM);
                              cached per device and size class (dtc_get_kernel_stats lists the
                              timings as autotune_* classes) */
  int32_t inner_precond;   /* preconditioner of the FP32 inner solve: 0 = Jacobi (as PETSc's
                              PCJACOBI), 1 = node-block Jacobi (3x3 diagonal blocks),
                              2 = multigrid V-cycle on halved voxel grids (HEX20 domains are
                              first coarsened to the HEX08 mesh of the same voxels) */
  int32_t tensor_estimator; /* how ff is formed from the solutions: 0 = projection of the
                              reaction forces (the reference, mod_struct_calcmat.f90:254-280),
                              error linear in the solve error; 1 = energy products
                              ff = vv^-T (U^T K U), equal at the exact solution, error quadratic */
  int32_t chunk_domains;   /* at most this many domains per device pass (0: as many as fit in
                              80% of the free device memory); the adjoint checkpoints the
                              displacements of every pass but the last to host memory */
  int32_t graph_chunks;    /* 0: each chunk of CG iterations is captured once and replayed as a
                              CUDA graph; 1: kernels are launched one by one */
  int32_t tc_wait_spins;   /* tensor-core kernels: polls of a round's completion barrier before
                              the kernel gives up and the call returns DTC_ERR_INTERNAL
                              (0 -> 2^26; < 0 -> no poll: every such wait gives up at once).
                              Only for testing that error path; the drain before tensor memory
                              is freed keeps the full bound */
  int32_t device_mesher;   /* 1: mesh the domains on the device (the reference numbering, bit
                              for bit the host planner's result); 0: on host threads */
  int32_t macro_order;     /* 'Element order on macro scale' (mod_dtc_main_subroutines.f90:498-508):
                              1 (or 0) = 8-node macro element, 24 load cases; 2 = 20-node macro
                              element, 60 load cases (init_displ_hexe20, mod_write_deck.f90:118-279;
                              the quadratic load-case matrix, mod_struct_calcmat.f90:1780-2028, with
                              its typing defects repaired; quad face sums :368-401).  Order 2 solves
                              the 60 load cases as three passes of 24 columns (with the energy
                              estimator the solutions of the first two stay on the device for the
                              60 x 60 Gram matrix), needs dtc_domain_out.macro2 on every record,
                              and has no adjoint (keep_displacements must be 0) */
} dtc_options;

typedef struct dtc_domain_in {
  int64_t L[3];            /* x_D: voxels per domain edge (mod_decomp.f90:290) */
  int64_t xa_n[3];         /* 1-based first voxel of the domain in the volume
                              (mod_struct_preprocess.f90:89-91) */
  int64_t domain_number;   /* copied to the output record */
  int32_t elem_type;       /* DTC_HEX08 or DTC_HEX20 (MICRO_ELMNT_TYPE) */
  int32_t phi_type;        /* bytes per gray value: 1, 2 or 4 (TYPE_RAW ik1/ik2/ik4) */
  const void* phi;         /* L0*L1*L2 signed gray values, x fastest */
  int64_t llimit;          /* BINARIZE_LO: voxel is bone iff phi >= llimit (mod_gen_quadmesh.f90:296) */
  const float* E_voxel;    /* optional per-voxel Young's modulus (MPa), L0*L1*L2, x fastest.
                              NULL: every element uses E, which is the reference behaviour */
  double delta[3];         /* SPACING: voxel edge (mm); must be equal in x, y, z */
  double phdsize[3];       /* SIZE_DOMAIN (mm); the element scale is a = phdsize(1)*delta(1) */
  double E;                /* YOUNG_MODULUS (MPa) */
  double nu;               /* POISSON_RATIO; all domains of one call share it */
  double rve_strain;       /* RVE_STRAIN: eps of the load-case matrix vv */
} dtc_domain_in;

/* The leaves of a macro order 2 record whose size differs from the 24-load-case record: the
 * reference sizes ff and the effective numerical stiffness no_lc x no_lc
 * (mod_struct_calcmat.f90:158-160,289-303) and solves no_lc = 60 load cases. */
typedef struct dtc_macro2_out {
  int64_t iters[60];       /* CG iterations per load case */
  double relres[60];       /* final ||D^-1 r|| / ||D^-1 b|| per load case */
  double ff[3600];         /* "Domain forces" ff(60,60), column-major */
  double kmacro[3600];     /* "Effective numerical stiffness" ff * vv^-1 (60 x 60) */
} dtc_macro2_out;

typedef struct dtc_domain_out {
  int32_t status;          /* DTC_DOMAIN_* */
  int32_t refine_steps;    /* mixed path: FP64 refinement steps taken */
  int64_t domain_number;
  int64_t ne, nn, nb;      /* elements, nodes, constrained nodes of the reference mesh */
  int64_t n_free_dof;      /* unconstrained DOFs the solver iterates on */
  int64_t iters[24];       /* CG iterations per load case (summed inner iterations for mixed) */
  double relres[24];       /* final ||D^-1 r|| / ||D^-1 b|| evaluated in FP64 */
  double ff[576];          /* "Domain forces" ff(24,24) */
  double kmacro[576];      /* "Effective numerical stiffness" ff * vv^-1 */
  double sym_k;            /* symmetry deviation max|A-A^T|/max|A| of kmacro */
  double c[36];            /* "Effective stiffness" fv * meps */
  double sym_c;
  double ee[36];           /* "Averaged Effective stiffness" (C + C^T)/2 */
  double sym_ee;
  double cr1_angle, cr1_n[3], cr1_aa[9], cr1_ee[36], cr1_crit;  /* CR1 (monotropic) */
  double cr2_angle, cr2_n[3], cr2_aa[9], cr2_ee[36], cr2_crit;  /* CR2 (orthotropic) */
  int32_t cr1_iters, cr2_iters;  /* refinement iterations jj */
  double density;          /* ne / (L0*L1*L2) (mod_struct_calcmat.f90:1642-1651) */
  double* displ;           /* optional (NULL to skip): 24 x 3nn displacements incl. boundary
                              values, load-case major, reference DOF numbering 3*(node-1)+comp;
                              room for 72*(L0+1)(L1+1)(L2+1) doubles (HEX08) or
                              72*(2L0+1)(2L1+1)(2L2+1) (HEX20) always suffices */
  double* force;           /* optional: 24 x 3nn reaction forces AA_org*u, same layout */
  dtc_macro2_out* macro2;  /* macro_order 2: caller-owned, required; receives iters, relres, ff and
                              kmacro, while the 24-sized fields above stay zero (displ/force then
                              hold 60 x 3nn values: room for 180*(grid nodes) doubles).  Ignored
                              for macro order 1 */
} dtc_domain_out;

typedef struct dtc_mesh_out {
  int64_t ne, nn, nb;      /* filled always */
  int32_t status;          /* DTC_DOMAIN_OK / EMPTY / NO_STRUCTURE / FEW_NODES */
  int32_t last_elem_partial; /* 1 when the mesher kept its last element although its region
                                was dropped (mod_gen_quadmesh.f90:598-613) */
  int64_t cap_elems, cap_nodes; /* capacities of the arrays below */
  int64_t* elems;          /* optional: elem_type*ne node ids, 1-based, 0 = dropped node */
  double* nodes;           /* optional: 3*nn coordinates */
  int64_t* bnode_ids;      /* optional: nb constrained node ids in node order */
  double* bnode_vals;      /* optional: nl x 3nb prescribed displacements, column-major, nl = 24
                              (macro order 1) or 60 (macro order 2) */
  int32_t macro_order;     /* in: macro element order of bnode_vals, 1 (or 0) or 2 */
  int32_t pad_;
} dtc_mesh_out;

typedef struct dtc_handle dtc_handle;

/* Version of this header the library was built with. */
int32_t dtc_abi_version(void);

/* Fill *opt with defaults: FP64, rtol 1e-3 and max_it 500000 (the reference's PETSc
 * options, f-src/mod_parameters.f90:23-32), rotation search on. */
void dtc_default_options(dtc_options* opt);

/* Create a solver bound to one CUDA device.  Replaces the per-domain
 * PetscInitialize/KSPCreate set-up of mod_dtc_main_subroutines.f90:144-148,995-1023. */
dtc_status dtc_create(dtc_handle** handle, const dtc_options* opt);

/* Release every device and host resource of the handle (PetscFinalize, :1220-1238). */
dtc_status dtc_destroy(dtc_handle* handle);

/* Mesh, solve and homogenise n domains.  Replaces, per domain, exec_single_domain's
 * generate_geometry (:247) + assembly (:516-579) + RHS/BC (:674-951) + 24 KSPSolve
 * (:1072-1078) + reactions (:1092-1123) + calc_effective_material_parameters (:1257).
 * in[i] and out[i] are caller-owned; out[i].displ/force may be NULL. */
dtc_status dtc_solve_batch(dtc_handle* handle, const dtc_domain_in* in, int64_t n,
                           dtc_domain_out* out);

/* Host-only: the reference mesh and boundary conditions of one domain (element order,
 * node numbering and constrained-node list bit-identical to gen_quadmesh_from_phi and
 * generate_boundaries).  Needs no device. */
dtc_status dtc_mesh_domain(const dtc_domain_in* in, dtc_mesh_out* out);

/* dtc_mesh_domain for n domains of one element type, computed on the handle's device
 * (gen_quadmesh_from_phi and generate_boundaries as device kernels: 26-connected regions by a
 * lock-free union-find, the bounding-box keep test, the compaction quirks, first-appearance
 * node numbering by prefix sums).  out[i] is filled exactly as dtc_mesh_domain fills it. */
dtc_status dtc_mesh_batch(dtc_handle* handle, const dtc_domain_in* in, int64_t n, dtc_mesh_out* out);

/* Host-only: element stiffness matrix of one voxel element, column-major (3*elem_type)^2,
 * node order of the mesher.  Mirrors Hexe08 / Hexe20 (f-src/mod_linfe.f90:161-776,
 * 890-4509), which tabulate it for a cube of edge a = phdsize(1)*delta(1) and modulus E. */
dtc_status dtc_element_stiffness(int32_t elem_type, double E, double a, double nu, double* ke);

/* Adjoint of the last dtc_solve_batch on this handle (which must have run with
 * keep_displacements = 1 and E_voxel given): for each domain i, dL/dE_voxel given
 * dL/dC = dloss_dc[36*i .. 36*i+35] (column-major 6x6, C = out.c).  Writes
 * L0*L1*L2 floats per domain into grad_e[i] (caller-owned).  No reference counterpart:
 * the reference has no gradient; this is the element-energy contraction
 * dff(r,lc)/dE_e = sum_a vv^-1(a,r) u_a,e^T (Ke/E) u_lc,e at the converged solution. */
dtc_status dtc_energy_grad(dtc_handle* handle, const double* dloss_dc, float* const* grad_e,
                           int64_t n);

/* dtc_solve_batch with the per-voxel moduli in device memory: E_voxel_dev[i] (n pointers in
 * host memory; NULL for a domain without per-voxel moduli) points to L0*L1*L2 floats on the
 * handle's device, x fastest; in[i].E_voxel is ignored for those domains.  The moduli are
 * copied once through a pinned host buffer owned by the handle (the host mesh planning and
 * multigrid build read them), then the call proceeds as dtc_solve_batch.  The copies are
 * ordered after work already submitted to the legacy default stream.  No reference
 * counterpart: the torch binding of the adjoint passes its tensors here. */
dtc_status dtc_solve_batch_device_moduli(dtc_handle* handle, const dtc_domain_in* in, int64_t n,
                                         dtc_domain_out* out, const float* const* E_voxel_dev);

/* dtc_energy_grad writing into device memory: grad_e_dev[i] (n pointers in host memory) points
 * to L0*L1*L2 floats on the handle's device; filled by device-to-device copies, complete when
 * the call returns.  No reference counterpart. */
dtc_status dtc_energy_grad_device(dtc_handle* handle, const double* dloss_dc, float* const* grad_e_dev,
                                  int64_t n);

/* Timing and work counters of the last dtc_solve_batch: device time of the solve in ms
 * (CUDA events on the solver stream, from the uploaded voxel factors to the last kernel,
 * summed over device passes; host meshing excluded), kernels launched, and the sum over
 * domains of free DOFs x load cases x CG iterations. */
dtc_status dtc_get_stats(const dtc_handle* handle, double* ms_solve, int64_t* kernel_launches,
                         double* dof_iterations);

/* Rotation search of given tensors (f-src/mod_struct_calcmat.f90:533-1603, criteria also
 * f-src/mod_tensor_opt.f90:40-603): the CR1/CR2 sweep and refinement on the handle's device,
 * then the angle, axis, frame and rotated tensor of each criterion on the host, exactly as
 * dtc_solve_batch does with rotation_search = 1.
 *   ee  : n x 36 doubles in host memory (6x6 column-major, symmetric: the "Averaged
 *         Effective stiffness" leaf)
 *   out : n records; only the cr1_* and cr2_* fields are written. */
dtc_status dtc_rotation_search(dtc_handle* handle, const double* ee, int64_t n, dtc_domain_out* out);

/* Rotation search (CR1/CR2 sweep and refinement, f-src/mod_struct_calcmat.f90:533-1603) on
 * tensors already in device memory, without allocating anything.  For callers that cannot
 * allocate device memory at the point of the call -- e.g. a host code that runs this step
 * while it captures a CUDA stream, or a host that hands the library only memory from its
 * own pool -- so the solver's usual per-call scratch allocation is not an option.
 * No counterpart in the reference.
 *   ee   : n x 36 doubles on the current device (6x6 column-major, symmetric)
 *   ang  : n x 2 x 3 int64 outputs: argmin angles (alpha, phi, eta) for CR1 then CR2, in
 *          units of 10^-jj degree
 *   jj   : n x 2 int32 outputs: refinement iterations;  crit: n x 2 doubles: final criterion
 *   stream: a cudaStream_t (NULL = default stream); work is stream-ordered, the call does
 *          not synchronise.
 * n must not exceed 1024: the scratch is one fixed 2 MiB device array per device, kept until
 * the process exits, shared by all calls; calls that overlap on the GPU race on it.
 * The first call on a device resolves that array's address and uploads two small tables
 * (unless dtc_solve_batch or dtc_rotation_search uploaded them already), then waits for the
 * device, so it should come before any stream capture.  The tables are written once per
 * device and process, never again, and the address is kept for the life of the process:
 * do not use this entry point across a cudaDeviceReset.  Sizes beyond the maximum return
 * DTC_ERR_INVALID_ARGUMENT. */
dtc_status dtc_rotation_search_noalloc(const double* ee, int64_t n, int64_t* ang, int32_t* jj, double* crit,
                                       void* stream);

/* Per kernel class of the last dtc_solve_batch (filled when profile_kernels = 1): launches,
 * summed CUDA-event time, and the algorithmic bytes / flops of one average launch. */
typedef struct dtc_kernel_stats {
  char name[32];
  int64_t launches;
  double ms_total;
  double bytes_per_launch;
  double flops_per_launch;
} dtc_kernel_stats;

/* Copies up to cap entries; *count receives the number of kernel classes. */
dtc_status dtc_get_kernel_stats(const dtc_handle* handle, dtc_kernel_stats* out, int32_t cap,
                                int32_t* count);

/* Message describing the last error on this handle (never NULL). */
const char* dtc_last_error(const dtc_handle* handle);

#ifdef __cplusplus
}
#endif
#endif /* DTC_H */
