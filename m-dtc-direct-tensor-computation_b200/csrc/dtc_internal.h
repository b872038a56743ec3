// dtc_internal.h -- shared definitions of the host planner and the sm_100a kernels.
//
// Device layout (one domain = one cubic control volume of L0 x L1 x L2 voxels):
//  * nodes live on the (m*L0+1)(m*L1+1)(m*L2+1) grid (m = 1: voxel corners, HEX08; m = 2: the
//    doubled grid carrying the HEX20 corner and mid-edge nodes), index n = x + nx*(y + ny*z);
//  * every nodal vector is [node][component][load case] with the 24 load cases innermost,
//    so the 24 right-hand sides of one DOF are one contiguous 96/192-byte run;
//  * per voxel one float modulus factor: E_voxel, or 1.0 when every element uses E; 0 for
//    void voxels and voxels the mesher dropped.  The FP64 per-domain factor D.scale (a * E,
//    or a; a = phdsize*delta, the reference's Ke scale) multiplies every operator output, so
//    no FP64 quantity passes through float rounding;
//  * per node one flag byte (active: touches a kept voxel; boundary: on the domain box).
// Work is cut into tiles of 8 x 4 x 4 nodes; a CTA of 128 threads handles one tile for
// 8 of the 24 load cases (1-D grid, the three load-case groups of a tile adjacent), each
// thread one (y,z) row of the tile and one load case, sweeping x with a 2-plane register
// window (the slab sweep of the HEX08 operator; the SIMT sweeps take their own lists of
// kSweepX-long rows, which halves the start-up of the window per node).  HEX20 uses voxel bricks (ebe.cuh); the
// multigrid CG vectors use a flat list of active interior nodes (mg.cuh).
#pragma once
#include <cstdint>

namespace dtc {

constexpr int kNLC = 24;          // load cases of the linear macro element
constexpr int kTileX = 8, kTileY = 4, kTileZ = 4;
constexpr int kSweepX = 16;       // nodes per row of the SIMT slab sweeps (own tile lists: two tiles in x)
constexpr int kLcGroup = 8;       // load cases per CTA
constexpr int kThreads = 128;     // 8 load cases x 16 rows

enum : uint8_t { kNodeActive = 1, kNodeBoundary = 2 };

struct DomDev {
  int32_t L[3];        // voxels per edge
  int32_t n[3];        // nodes per edge: m*L+1
  int32_t m;           // node-grid refinement: 1 (HEX08 corners), 2 (HEX20 corners + mid-edges)
  int32_t pad_;
  int64_t vox_off;     // offset into the voxel scale array
  int64_t node_off;    // offset into node arrays (vectors are node_off*72)
  int64_t min_c_off[3];  // xa_n - 1: node (i,j,k) sits at ((i,j,k) + min_c_off) * delta
  double delta;        // voxel edge
  double scale;        // per-domain stiffness factor: a (= phdsize*delta) times E when the
                       // voxel array holds 1.0 for a constant modulus
  double min_c[3];     // domain box (mod_struct_preprocess.f90:516-517)
  double max_c[3];
};

struct Tile {
  int32_t dom;
  int16_t x0, y0, z0;
  int16_t pad;
};

// Per (domain, load case) state of the Jacobi-PCG recurrence (PETSc KSPSolve_CG).
struct ColState {
  double beta, betaold, dpi, bfac, dp0, ttol, dp;
  int32_t its, reason, active, pad;
};

// reasons (KSPConvergedReason analogues)
enum : int32_t { kIterating = 0, kConverged = 2, kConvergedAtol = 3, kDivergedIts = -3,
                 kDivergedDtol = -4, kIndefinite = -8, kNanOrInf = -9 };

// -------------------------------------------------------------------------------------
// Host-side launchers (kernels.cu)
struct DevBatch;  // opaque device-side batch (kernels.cu)

}  // namespace dtc
