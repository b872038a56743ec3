// kernels.cu -- sm_100a kernels of the batched voxel solver and its host driver.
//
// Operator: the assembled stiffness of the reference (MatSetValues of one Ke per element,
// f-src/mod_dtc_main_subroutines.f90:516-579) is never formed.  HEX08: K*u is applied
// matrix-free as a node-centric sweep: the output at node n sums, over the <= 8 kept voxels
// around n, s_v * Khat[rows of n's corner, :] * u_v, where s_v = E_v * a and Khat the unit
// voxel stiffness.  HEX20: element-by-element on voxel bricks staged in shared memory
// (ebe.cuh), nodes on the doubled grid.  Constrained DOFs (all nodes on the domain box, mod_struct_preprocess.f90:
// 564-592) are excluded from the unknowns exactly like MatZeroRowsColumns with diag 0
// (:945-951), so the iteration runs on the interior nodes only.
//
// Solver: per (domain, load case) the Jacobi-PCG recurrence of PETSc's KSPSolve_CG with
// KSPConvergedDefault (zero initial guess, preconditioned 2-norm, ttol = max(rtol*||D^-1 b||,
// 1e-50), divergence at 1e5*||D^-1 b||) -- four launches per iteration for the whole batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <map>
#include <mutex>
#include <tuple>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "fe.h"
#include "kernels.cuh"
#include "solver.h"

namespace dtc {

__constant__ double c_khat64[576];   // unit voxel stiffness, column-major (symmetric)
__constant__ float c_khat32[576];
// the 24 load-case columns of the current column pass of the macro modes for eps = 1e-6:
// uu(nm,3,24) column-major, nm = 8 (macro order 1) or 20 (macro order 2); columns past the
// last load case are zero
__constant__ double c_uu[20 * 3 * kNLC];
__constant__ double c_k20_64[3600];       // unit HEX20 element matrix (ring node order)

template <typename T> struct KhatC;
template <> struct KhatC<float> {
  static __device__ __forceinline__ float at(int i) { return c_khat32[i]; }
};
template <> struct KhatC<double> {
  static __device__ __forceinline__ double at(int i) { return c_khat64[i]; }
};

// -------------------------------------------------------------------------------------
// HEX08: matrix-free K*u on node rows (the default SIMT operator of the corner grid).  A thread
// owns one (y, z) row of a tile for one load case and sweeps x.  Between node planes x and x+1
// lie the 4 voxels (x, y-1..y, z-1..z) of the row; each kept voxel contributes
// s_v * Khat[rows of its corner, :] * u_v to node x (corner with offset 0 in x) and to node x+1
// (offset 1), both from one read of its 8 corner values (voxel_rp / voxel_rd below).  FIRST: the
// slab left of the tile, whose contribution to the first node only is needed.

template <bool GUARD>
__device__ __forceinline__ void load_voxels(float (&sp)[2][2], const float* __restrict__ svox, const DomDev& D, int vx,
                                            int y, int z) {
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int vy = y - 1 + b, vz = z - 1 + c;
      bool ok = true;
      if (GUARD) ok = (vx >= 0 && vx < D.L[0] && vy >= 0 && vy < D.L[1] && vz >= 0 && vz < D.L[2]);
      const int64_t off = ok ? vx + (int64_t)D.L[0] * (vy + (int64_t)D.L[1] * vz) : 0;
      sp[b][c] = ok ? __ldg(svox + D.vox_off + off) : 0.0f;
    }
}

// FP32 slab on packed two-lane FMAs (sm_100 FFMA2).  A voxel of the row feeds two output rows
// r of the thread's nodes: the corner at plane x (l0, node x) and the corner at plane x+1 (l1,
// node x+1); one packed FMA applies both rows' entries of a column to one broadcast input value
// (lane x: node x, lane y: node x+1), halving the FMA instructions of the scalar slab (voxel_rp).
// The table holds the two rows' entries side by side, per voxel slot (b, c) of the row.
__constant__ float2 c_khat32r2[4 * 3 * 24];   // [2b + c][r][col] = (Khat[3 l0 + r, col], Khat[3 l1 + r, col])

// Voxel-outer FP32 slab (the FP32 sweeps): the kept voxel (b, c) of the row between planes x
// (rp: the row's values at plane x for its load case) and x+1 reads its own 8 corners' 24 values
// (mostly L1 hits: neighbouring rows and voxels share them) and applies them with packed FMAs.
// No node plane stays in registers between steps, which keeps a thread at 64-80 registers (6 or
// 8 CTAs per SM) where a window of two node planes in registers needed ~100.
template <bool FIRST>
__device__ __forceinline__ void voxel_rp(const float* __restrict__ rp, int sy, int sz, int b, int c, float s,
                                         float (&cur)[3], float (&nxt)[3]) {
  float2 acc[3];
#pragma unroll
  for (int r = 0; r < 3; ++r) acc[r] = make_float2(0.f, 0.f);
#pragma unroll
  for (int mz = 0; mz < 2; ++mz)
#pragma unroll
    for (int my = 0; my < 2; ++my)
#pragma unroll
      for (int mx = 0; mx < 2; ++mx) {
        const int lm = corner_local(mx, my, mz);
        const float* q = rp + mx * (3 * kNLC) + (b - 1 + my) * sy + (c - 1 + mz) * sz;
#pragma unroll
        for (int cj = 0; cj < 3; ++cj) {
          const float v = __ldg(q + cj * kNLC);
          const float2 vv = make_float2(v, v);
#pragma unroll
          for (int r = 0; r < 3; ++r)
            acc[r] = __ffma2_rn(c_khat32r2[((2 * b + c) * 3 + r) * 24 + 3 * lm + cj], vv, acc[r]);
        }
      }
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    if (!FIRST) cur[r] = fmaf(s, acc[r].x, cur[r]);
    nxt[r] = fmaf(s, acc[r].y, nxt[r]);
  }
}
template <bool FIRST>
__device__ __forceinline__ void row_slab(const float* __restrict__ rp, int sy, int sz, const float (&sv)[2][2],
                                         float (&cur)[3], float (&nxt)[3]) {
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int c = 0; c < 2; ++c)
      if (sv[b][c] != 0.0f) voxel_rp<FIRST>(rp, sy, sz, b, c, sv[b][c], cur, nxt);
}

// Voxel-outer FP64 slab (scalar FMAs, the summation order of slab): the kept voxel (b, c) of
// the row between planes x and x+1 reads its 8 corners' values from u, kb being the index of the
// row's value at plane x for its load case (negative when the row starts left of the grid: a
// voxel inside the grid has all its corners inside it, so only kept voxels' corners are read).
template <bool FIRST>
__device__ __forceinline__ void voxel_rd(const double* __restrict__ u, int64_t kb, int sy, int sz, int b, int c,
                                         float s, double (&cur)[3], double (&nxt)[3]) {
  const int l0 = corner_local(0, 1 - b, 1 - c), l1 = corner_local(1, 1 - b, 1 - c);
  double t0 = 0, t1 = 0, t2 = 0, q0 = 0, q1 = 0, q2 = 0;
#pragma unroll 1
  for (int mz = 0; mz < 2; ++mz)
#pragma unroll
    for (int my = 0; my < 2; ++my)
#pragma unroll
      for (int mx = 0; mx < 2; ++mx) {
        const int lm = corner_local(mx, my, mz);
        const int64_t k = kb + mx * (3 * kNLC) + (b - 1 + my) * sy + (c - 1 + mz) * sz;
#pragma unroll
        for (int cj = 0; cj < 3; ++cj) {
          const double v = __ldg(u + k + cj * kNLC);
          const int col = 24 * (3 * lm + cj);
          if (!FIRST) {
            t0 = fma(KhatC<double>::at(col + 3 * l0 + 0), v, t0);
            t1 = fma(KhatC<double>::at(col + 3 * l0 + 1), v, t1);
            t2 = fma(KhatC<double>::at(col + 3 * l0 + 2), v, t2);
          }
          q0 = fma(KhatC<double>::at(col + 3 * l1 + 0), v, q0);
          q1 = fma(KhatC<double>::at(col + 3 * l1 + 1), v, q1);
          q2 = fma(KhatC<double>::at(col + 3 * l1 + 2), v, q2);
        }
      }
  const double ts = (double)s;
  if (!FIRST) {
    cur[0] = fma(ts, t0, cur[0]);
    cur[1] = fma(ts, t1, cur[1]);
    cur[2] = fma(ts, t2, cur[2]);
  }
  nxt[0] = fma(ts, q0, nxt[0]);
  nxt[1] = fma(ts, q1, nxt[1]);
  nxt[2] = fma(ts, q2, nxt[2]);
}
template <bool FIRST>
__device__ __forceinline__ void row_slab_d(const double* __restrict__ u, int64_t kb, int sy, int sz,
                                           const float (&sv)[2][2], double (&cur)[3], double (&nxt)[3]) {
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int c = 0; c < 2; ++c)
      if (sv[b][c] != 0.0f) voxel_rd<FIRST>(u, kb, sy, sz, b, c, sv[b][c], cur, nxt);
}


// The 4 voxels of an interior node row between planes x and x+1 (the sweeps over interior
// rows): a pointer that advances by one voxel per plane, 32-bit offsets of the y and z neighbours.
struct VoxRow {
  const float* p;
  int sy, sz;
  __device__ __forceinline__ void start(const float* __restrict__ svox, const DomDev& D, int vx, int y, int z) {
    sy = D.L[0];
    sz = D.L[0] * D.L[1];
    p = svox + D.vox_off + vx + (int64_t)D.L[0] * ((y - 1) + (int64_t)D.L[1] * (z - 1));
  }
  __device__ __forceinline__ void load(float (&sp)[2][2]) const {
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int c = 0; c < 2; ++c) sp[b][c] = __ldg(p + b * sy + c * sz);
  }
};

// y = scale * K u on the tile's nodes.  ALL = false: interior nodes only (inputs are
// in-bounds without guards), optional dot accumulation acc[col] += u.y.  ALL = true: every
// node of the grid (reaction forces; only the voxel factors need guards, since a voxel inside the
// grid has all its corners inside it).  FP32 rows use voxel_rp, FP64 rows voxel_rd.  xlen: nodes per row of the tile list (kTileX or
// kSweepX).  bnd_only: u vanishes off the domain box (the boundary
// values before the first solve) and y is zero on entry; a row whose neighbour rows lie
// inside the box then only has nonzero output at x = 1 and x = n0 - 2, and computes only those.
// MINB: CTAs per SM the register allocation is sized for; FP32 6 (at most 80 registers) or 8 (64),
// FP64 4 (128) or 6 (80), chosen per batch class by the sweep autotuner
template <typename T, bool ALL, bool DOT, int MINB = (sizeof(T) == 4 ? 6 : 4)>
__global__ void __launch_bounds__(kThreads, MINB) k_matvec(const Tile* __restrict__ tiles,
                                                                          const DomDev* __restrict__ doms,
                                                     const float* __restrict__ svox, const T* __restrict__ u,
                                                     T* __restrict__ y, double scale, double* __restrict__ acc,
                                                     const int* __restrict__ dom_active, int bnd_only, int xlen) {
  __shared__ double red[32];
  const Tile t = tiles[blockIdx.x / 3];
  if (dom_active && !dom_active[t.dom]) return;
  const DomDev D = doms[t.dom];
  const int lc = (blockIdx.x % 3) * kLcGroup + (threadIdx.x & 7);
  const int row = threadIdx.x >> 3;
  const int yy = t.y0 + (row & 3), zz = t.z0 + (row >> 2);
  const int lo = ALL ? 0 : 1;
  const int xhi = ALL ? D.n[0] - 1 : D.n[0] - 2, yhi = ALL ? D.n[1] - 1 : D.n[1] - 2, zhi = ALL ? D.n[2] - 1 : D.n[2] - 2;
  // nodes x0 .. xe of the row, x0 from the tile start
  int x0 = t.x0, xe = min(xhi, t.x0 + xlen - 1);
  if (!ALL && bnd_only && yy >= 2 && yy <= D.n[1] - 3 && zz >= 2 && zz <= D.n[2] - 3) {
    const bool has_lo = x0 <= 1 && 1 <= xe, has_hi = x0 <= D.n[0] - 2 && D.n[0] - 2 <= xe;
    if (has_lo && !has_hi) xe = 1;
    else if (has_hi && !has_lo) x0 = D.n[0] - 2;
    else if (!has_lo) xe = x0 - 1;   // neither: nothing to compute on this row
  }
  double dot = 0.0;
  if constexpr (!ALL && sizeof(T) == 4) {
    if (yy >= lo && yy <= yhi && zz >= lo && zz <= zhi && x0 <= xe) {
      const int sy = D.n[0] * (3 * kNLC), sz = D.n[0] * D.n[1] * (3 * kNLC);
      const float* rp = u + vec_index(node_index(D, x0 - 1, yy, zz), 0, lc);   // plane x0 - 1
      VoxRow V;
      float sv[2][2];
      float cur[3] = {0.f, 0.f, 0.f}, nxt[3] = {0.f, 0.f, 0.f};
      V.start(svox, D, x0 - 1, yy, zz);
      V.load(sv);
      bool anyp = (sv[0][0] != 0.f) | (sv[0][1] != 0.f) | (sv[1][0] != 0.f) | (sv[1][1] != 0.f);
      row_slab<true>(rp, sy, sz, sv, cur, nxt);
#pragma unroll 1
      for (int x = x0; x <= xe; ++x) {
        rp += 3 * kNLC;   // plane x
        ++V.p;
        V.load(sv);
        const bool anyc = (sv[0][0] != 0.f) | (sv[0][1] != 0.f) | (sv[1][0] != 0.f) | (sv[1][1] != 0.f);
#pragma unroll
        for (int c = 0; c < 3; ++c) { cur[c] = nxt[c]; nxt[c] = 0.f; }
        row_slab<false>(rp, sy, sz, sv, cur, nxt);
        if (anyp | anyc) {
          const int64_t b = rp - u;
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float v = (float)(scale * D.scale * (double)cur[c]);
            y[b + c * kNLC] = v;
            if (DOT) dot += (double)__ldg(rp + c * kNLC) * (double)v;
          }
        }
        anyp = anyc;
      }
    }
  } else if (yy >= lo && yy <= yhi && zz >= lo && zz <= zhi && x0 <= xe) {
    // FP64: voxel-outer slab; ALL rows may lie on the domain box, where only the voxel factors
    // need guards (out-of-grid voxels read as void)
    const int sy = D.n[0] * (3 * kNLC), sz = D.n[0] * D.n[1] * (3 * kNLC);
    int64_t kx = vec_index(node_index(D, x0 - 1, yy, zz), 0, lc);   // plane x0 - 1 of the row
    VoxRow V;
    float sv[2][2];
    double cur[3] = {0, 0, 0}, nxt[3] = {0, 0, 0};
    if constexpr (ALL) {
      load_voxels<true>(sv, svox, D, x0 - 1, yy, zz);
    } else {
      V.start(svox, D, x0 - 1, yy, zz);
      V.load(sv);
    }
    bool anyp = (sv[0][0] != 0.f) | (sv[0][1] != 0.f) | (sv[1][0] != 0.f) | (sv[1][1] != 0.f);
    row_slab_d<true>(u, kx, sy, sz, sv, cur, nxt);
#pragma unroll 1
    for (int x = x0; x <= xe; ++x) {
      kx += 3 * kNLC;   // plane x
      if constexpr (ALL) {
        load_voxels<true>(sv, svox, D, x, yy, zz);
      } else {
        ++V.p;
        V.load(sv);
      }
      const bool anyc = (sv[0][0] != 0.f) | (sv[0][1] != 0.f) | (sv[1][0] != 0.f) | (sv[1][1] != 0.f);
#pragma unroll
      for (int c = 0; c < 3; ++c) { cur[c] = nxt[c]; nxt[c] = 0.0; }
      row_slab_d<false>(u, kx, sy, sz, sv, cur, nxt);
      if (anyp | anyc) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const double v = scale * D.scale * cur[c];
          y[kx + c * kNLC] = v;
          if (DOT) dot += __ldg(u + kx + c * kNLC) * v;
        }
      }
      anyp = anyc;
    }
  }
  if (DOT) {
    const double s = block_sum_lc<double>(dot, red);
    if (threadIdx.x < 8) atomicAdd(acc + (int64_t)t.dom * kNLC + lc, s);
  }
}

}  // namespace dtc

#include "ebe.cuh"
#include "mg.cuh"

namespace dtc {

// -------------------------------------------------------------------------------------
// Node set-up: flags, the Jacobi diagonal sum_v s_v Ke(ii) (PCJACOBI of the row-and-column-
// zeroed matrix; constrained rows are never iterated on) and the node-block inverse.  One
// thread per node of the (fine) grid.  Adjacent voxels of a node: per axis, a coordinate f
// lies in voxel f/m - 1 (local offset m) and f/m (offset 0) when f is a multiple of m, else
// only in (f-1)/2 (offset 1, HEX20 mid-edge).
template <int NEN> __device__ __forceinline__ int local_node(int ox, int oy, int oz);
template <> __device__ __forceinline__ int local_node<8>(int ox, int oy, int oz) { return corner_local(ox, oy, oz); }
template <> __device__ __forceinline__ int local_node<20>(int ox, int oy, int oz) {
  for (int a = 0; a < 20; ++a)
    if (kRingOff[a][0] == ox && kRingOff[a][1] == oy && kRingOff[a][2] == oz) return a;
  return -1;
}
template <int NEN> __device__ __forceinline__ double ke64(int i);
template <> __device__ __forceinline__ double ke64<8>(int i) { return c_khat64[i]; }
template <> __device__ __forceinline__ double ke64<20>(int i) { return c_k20_64[i]; }

template <int NEN>
__global__ void __launch_bounds__(kThreads) k_node_setup(const Tile* __restrict__ tiles, const DomDev* __restrict__ doms,
                                                         const float* __restrict__ svox, uint8_t* __restrict__ flags,
                                                         double* __restrict__ dinv64, float* __restrict__ dinv32,
                                                         float* __restrict__ binv32) {
  constexpr int ND = 3 * NEN;
  const Tile t = tiles[blockIdx.x];
  const DomDev D = doms[t.dom];
  const int x = t.x0 + (threadIdx.x & 7), row = threadIdx.x >> 3;
  const int y = t.y0 + (row & 3), z = t.z0 + (row >> 2);
  if (x >= D.n[0] || y >= D.n[1] || z >= D.n[2]) return;
  const int m = D.m;
  const int f[3] = {x, y, z};
  int vc[3][2], oc[3][2], nc[3];
  for (int d = 0; d < 3; ++d) {
    if (f[d] % m == 0) { nc[d] = 2; vc[d][0] = f[d] / m - 1; oc[d][0] = m; vc[d][1] = f[d] / m; oc[d][1] = 0; }
    else { nc[d] = 1; vc[d][0] = (f[d] - 1) / 2; oc[d][0] = 1; }
  }
  double d3[3] = {0, 0, 0};
  double blk[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  bool active = false;
  for (int i = 0; i < nc[0]; ++i)
    for (int j = 0; j < nc[1]; ++j)
      for (int k = 0; k < nc[2]; ++k) {
        const int vx = vc[0][i], vy = vc[1][j], vz = vc[2][k];
        if (vx < 0 || vy < 0 || vz < 0 || vx >= D.L[0] || vy >= D.L[1] || vz >= D.L[2]) continue;
        const float s = svox[D.vox_off + vx + (int64_t)D.L[0] * (vy + (int64_t)D.L[1] * vz)];
        if (s == 0.0f) continue;
        const int ln = local_node<NEN>(oc[0][i], oc[1][j], oc[2][k]);
        if (ln < 0) continue;
        active = true;
        for (int a = 0; a < 3; ++a) d3[a] += (double)s * ke64<NEN>((3 * ln + a) * (ND + 1));
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) blk[a][b] += (double)s * ke64<NEN>((3 * ln + a) + ND * (3 * ln + b));
      }
  for (int a = 0; a < 3; ++a) d3[a] *= D.scale;
  const bool bnd = (x == 0 || x == D.n[0] - 1 || y == 0 || y == D.n[1] - 1 || z == 0 || z == D.n[2] - 1);
  const int64_t n = node_index(D, x, y, z);
  flags[n] = (active ? kNodeActive : 0) | (bnd ? kNodeBoundary : 0);
  for (int a = 0; a < 3; ++a) {
    const double di = (active && !bnd && d3[a] != 0.0) ? 1.0 / d3[a] : 0.0;
    dinv64[n * 3 + a] = di;
    dinv32[n * 3 + a] = (float)di;
  }
  float bi[6] = {0, 0, 0, 0, 0, 0};
  if (active && !bnd) {
    const double a = blk[0][0], b = blk[0][1], c = blk[0][2], e = blk[1][1], ff = blk[1][2], g = blk[2][2];
    const double c00 = e * g - ff * ff, c01 = c * ff - b * g, c02 = b * ff - c * e;
    const double det = a * c00 + b * c01 + c * c02;
    if (det > 0.0) {
      const double inv = 1.0 / (det * D.scale);
      bi[0] = (float)(c00 * inv);
      bi[1] = (float)((a * g - c * c) * inv);
      bi[2] = (float)((a * e - b * b) * inv);
      bi[3] = (float)(c01 * inv);
      bi[4] = (float)(c02 * inv);
      bi[5] = (float)((b * c - a * ff) * inv);
    }
  }
  for (int k = 0; k < 6; ++k) binv32[n * 6 + k] = bi[k];
}

// Preconditioner z = M^-1 r for the 3 components of one node: scalar Jacobi (PETSc PCJACOBI)
// or node-block Jacobi (inverse 3x3 diagonal block, symmetric storage).
template <typename T, bool BLOCK>
__device__ __forceinline__ void precond(const T* __restrict__ m, int64_t n, const T (&r)[3], T (&z)[3]) {
  if (BLOCK) {
    const T* b = m + n * 6;
    z[0] = b[0] * r[0] + b[3] * r[1] + b[4] * r[2];
    z[1] = b[3] * r[0] + b[1] * r[1] + b[5] * r[2];
    z[2] = b[4] * r[0] + b[5] * r[1] + b[2] * r[2];
  } else {
    z[0] = m[n * 3 + 0] * r[0];
    z[1] = m[n * 3 + 1] * r[1];
    z[2] = m[n * 3 + 2] * r[2];
  }
}

// Prescribed displacements of every load case on the boundary nodes
// (determine_prescribed_displ, mod_write_deck.f90:22-51): sum_l N_l(xi(x)) uu(l,c,lc).
__device__ __forceinline__ void node_xi(const DomDev& D, int x, int y, int z, double xi[3]) {
  const int g[3] = {x, y, z};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double pos = D.m == 1 ? (double)((int64_t)g[k] + (int64_t)D.min_c_off[k]) * D.delta
                                : ((double)g[k] / (double)D.m + (double)D.min_c_off[k]) * D.delta;
    xi[k] = 2.0 / (D.max_c[k] - D.min_c[k]) * pos - (D.max_c[k] + D.min_c[k]) / (D.max_c[k] - D.min_c[k]);
  }
}
__device__ __forceinline__ void shape8(const double xi[3], double N[8]) {
  const double g1x = 0.5 * (1.0 - xi[0]), g2x = 0.5 * (1.0 + xi[0]);
  const double g1y = 0.5 * (1.0 - xi[1]), g2y = 0.5 * (1.0 + xi[1]);
  const double g1z = 0.5 * (1.0 - xi[2]), g2z = 0.5 * (1.0 + xi[2]);
  N[0] = g1x * g1y * g1z; N[1] = g2x * g1y * g1z; N[2] = g2x * g2y * g1z; N[3] = g1x * g2y * g1z;
  N[4] = g1x * g1y * g2z; N[5] = g2x * g1y * g2z; N[6] = g2x * g2y * g2z; N[7] = g1x * g2y * g2z;
}

// ANSYS 20-node macro shape functions, as the host's macro_shape20 (phi_NN_hexe20,
// mod_linfe.f90:827-888)
__device__ __forceinline__ void shape20(const double xi[3], double N[20]) {
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
template <int NM>
__device__ __forceinline__ void macro_shape_dev(const double xi[3], double (&N)[NM]) {
  if constexpr (NM == 20) shape20(xi, N);
  else shape8(xi, N);
}

// Prescribed values of the current column pass on the domain-box nodes: component c of load
// case lc is sum_l N_l(xi(x)) uu(l, c, lc) (determine_prescribed_displ, mod_write_deck.f90:22-51).
template <int NM>
__global__ void __launch_bounds__(kThreads) k_boundary_values(const Tile* __restrict__ tiles,
                                                              const DomDev* __restrict__ doms,
                                                              const uint8_t* __restrict__ flags,
                                                              double* __restrict__ X) {
  const Tile t = tiles[blockIdx.x];
  const DomDev D = doms[t.dom];
  const int x = t.x0 + (threadIdx.x & 7), row = threadIdx.x >> 3;
  const int y = t.y0 + (row & 3), z = t.z0 + (row >> 2);
  if (x >= D.n[0] || y >= D.n[1] || z >= D.n[2]) return;
  const int64_t n = node_index(D, x, y, z);
  const uint8_t f = flags[n];
  if (!(f & kNodeActive) || !(f & kNodeBoundary)) return;
  double xi[3], N[NM];
  node_xi(D, x, y, z, xi);
  macro_shape_dev<NM>(xi, N);
  for (int c = 0; c < 3; ++c)
    for (int lc = 0; lc < kNLC; ++lc) {
      double s = 0.0;
      for (int l = 0; l < NM; ++l) s += N[l] * c_uu[l + NM * c + 3 * NM * lc];
      X[vec_index(n, c, lc)] = s;
    }
}

// -------------------------------------------------------------------------------------
// CG vector kernels on interior tiles; lane = load case, row = (y,z), sweep x.
#define DTC_TILE_PROLOGUE                                                      \
  const Tile t = tiles[blockIdx.x / 3];                                        \
  if (dom_active && !dom_active[t.dom]) return;                                \
  const DomDev D = doms[t.dom];                                                \
  const int lc = (blockIdx.x % 3) * kLcGroup + (threadIdx.x & 7);              \
  const int row = threadIdx.x >> 3;                                            \
  const int yy = t.y0 + (row & 3), zz = t.z0 + (row >> 2);                     \
  const bool rowok = yy >= 1 && yy <= D.n[1] - 2 && zz >= 1 && zz <= D.n[2] - 2; \
  const int64_t col = (int64_t)t.dom * kNLC + lc;

// p = M^-1 r + bfac * p
template <typename T, bool BLOCK>
__global__ void __launch_bounds__(kThreads) k_direction(const Tile* __restrict__ tiles, const DomDev* __restrict__ doms,
                                                        const uint8_t* __restrict__ flags, const T* __restrict__ dinv,
                                                        const T* __restrict__ r, T* __restrict__ p,
                                                        const ColState* __restrict__ st,
                                                        const int* __restrict__ dom_active) {
  DTC_TILE_PROLOGUE
  if (!rowok || !st[col].active) return;
  const T bf = (T)st[col].bfac;
  for (int i = 0; i < kTileX; ++i) {
    const int x = t.x0 + i;
    if (x > D.n[0] - 2) break;
    const int64_t n = node_index(D, x, yy, zz);
    if (!(flags[n] & kNodeActive)) continue;
    const int64_t k0 = vec_index(n, 0, lc);
    T rr[3], z[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) rr[c] = r[k0 + c * kNLC];
    precond<T, BLOCK>(dinv, n, rr, z);
#pragma unroll
    for (int c = 0; c < 3; ++c) p[k0 + c * kNLC] = z[c] + bf * p[k0 + c * kNLC];
  }
}

// x += alpha p ; r -= alpha w ; z = M^-1 r ; acc_zz += z.z ; acc_zr += z.r
// alpha = beta / (p.w) unless the column stopped or p.w flags an indefinite operator.
template <typename T, bool BLOCK>
__global__ void __launch_bounds__(kThreads) k_update(const Tile* __restrict__ tiles, const DomDev* __restrict__ doms,
                                                     const uint8_t* __restrict__ flags, const T* __restrict__ dinv,
                                                     T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p,
                                                     const T* __restrict__ w, const ColState* __restrict__ st,
                                                     const double* __restrict__ acc_pw, double* __restrict__ acc_zz,
                                                     double* __restrict__ acc_zr, const int* __restrict__ dom_active) {
  __shared__ double red[32];
  DTC_TILE_PROLOGUE
  double zz2 = 0.0, zr = 0.0;
  const ColState s = st[col];
  const double pw = acc_pw[col];
  const bool flip = s.its > 0 && ((pw > 0) != (s.dpi > 0) || pw == 0.0);
  const bool valid = s.active && pw != 0.0 && !flip;
  if (rowok && valid) {
    const T a = (T)(s.beta / pw);
    for (int i = 0; i < kTileX; ++i) {
      const int xx = t.x0 + i;
      if (xx > D.n[0] - 2) break;
      const int64_t n = node_index(D, xx, yy, zz);
      if (!(flags[n] & kNodeActive)) continue;
      const int64_t k0 = vec_index(n, 0, lc);
      T rn[3], z[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const int64_t k = k0 + c * kNLC;
        x[k] = x[k] + a * p[k];
        rn[c] = r[k] - a * w[k];
        r[k] = rn[c];
      }
      precond<T, BLOCK>(dinv, n, rn, z);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        zz2 += (double)z[c] * (double)z[c];
        zr += (double)z[c] * (double)rn[c];
      }
    }
  }
  const double s1 = block_sum_lc<double>(zz2, red);
  __syncthreads();
  const double s2 = block_sum_lc<double>(zr, red);
  if (threadIdx.x < 8 && valid) {
    atomicAdd(acc_zz + col, s1);
    atomicAdd(acc_zr + col, s2);
  }
}

// z = M^-1 r; acc_zz += z.z ; acc_zr += z.r (start of a solve)
template <typename T, bool BLOCK>
__global__ void __launch_bounds__(kThreads) k_initial_dots(const Tile* __restrict__ tiles,
                                                           const DomDev* __restrict__ doms,
                                                           const uint8_t* __restrict__ flags,
                                                           const T* __restrict__ dinv, const T* __restrict__ r,
                                                           double* __restrict__ acc_zz, double* __restrict__ acc_zr,
                                                           const int* __restrict__ dom_active) {
  __shared__ double red[32];
  DTC_TILE_PROLOGUE
  double zz2 = 0.0, zr = 0.0;
  if (rowok) {
    for (int i = 0; i < kTileX; ++i) {
      const int xx = t.x0 + i;
      if (xx > D.n[0] - 2) break;
      const int64_t n = node_index(D, xx, yy, zz);
      if (!(flags[n] & kNodeActive)) continue;
      const int64_t k0 = vec_index(n, 0, lc);
      T rn[3], z[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) rn[c] = r[k0 + c * kNLC];
      precond<T, BLOCK>(dinv, n, rn, z);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        zz2 += (double)z[c] * (double)z[c];
        zr += (double)z[c] * (double)rn[c];
      }
    }
  }
  const double s1 = block_sum_lc<double>(zz2, red);
  __syncthreads();
  const double s2 = block_sum_lc<double>(zr, red);
  if (threadIdx.x < 8) {
    atomicAdd(acc_zz + col, s1);
    atomicAdd(acc_zr + col, s2);
  }
}

// Column state at the start of a solve (KSPSolve_CG before its loop + KSPConvergedDefault
// at n = 0).  ttol = max(rtol * dp0, floor[col]) with floor = 1e-50 (abstol) when absent.
__global__ void k_colstate_init(ColState* __restrict__ st, double* __restrict__ acc_zz, double* __restrict__ acc_zr,
                                int* __restrict__ dom_active, double rtol, const double* __restrict__ floor_abs,
                                float* __restrict__ dirf) {
  const int d = blockIdx.x, lc = threadIdx.x;
  int act = 0;
  if (lc < kNLC) {
    const int64_t col = (int64_t)d * kNLC + lc;
    ColState s;
    const double dp0 = sqrt(acc_zz[col]);
    s.dp0 = dp0; s.dp = dp0; s.its = 0; s.bfac = 0.0; s.dpi = 0.0; s.betaold = 1.0; s.beta = 0.0; s.pad = 0;
    const double fl = floor_abs ? fmax(floor_abs[col], 1e-50) : 1e-50;
    s.ttol = fmax(rtol * dp0, fl);
    s.active = 0;
    if (!isfinite(dp0)) s.reason = kNanOrInf;
    else if (dp0 <= s.ttol) s.reason = kConverged;
    else {
      s.beta = acc_zr[col];
      if (s.beta == 0.0) { s.its = 1; s.reason = kConvergedAtol; }
      else { s.reason = kIterating; s.active = 1; }
    }
    st[col] = s;
    if (dirf) dirf[col] = s.active ? (float)s.bfac : NAN;
    acc_zz[col] = 0.0; acc_zr[col] = 0.0;
    act = s.active;
  }
  act = __syncthreads_or(act);
  if (threadIdx.x == 0) dom_active[d] = act;
}

// End of one CG iteration for every column (the tail of KSPSolve_CG's loop body).
__global__ void k_colstate(ColState* __restrict__ st, double* __restrict__ acc_pw, double* __restrict__ acc_zz,
                           double* __restrict__ acc_zr, int* __restrict__ dom_active, int64_t max_it,
                           float* __restrict__ dirf) {
  const int d = blockIdx.x, lc = threadIdx.x;
  int act = 0;
  if (lc < kNLC) {
    const int64_t col = (int64_t)d * kNLC + lc;
    ColState s = st[col];
    if (s.active) {
      const double pw = acc_pw[col];
      const bool flip = s.its > 0 && ((pw > 0) != (s.dpi > 0));
      s.its += 1;
      if (pw == 0.0 || flip) { s.reason = kIndefinite; s.active = 0; }
      else {
        s.dpi = pw;
        s.betaold = s.beta;
        const double dp = sqrt(acc_zz[col]);
        s.dp = dp;
        if (!isfinite(dp)) { s.reason = kNanOrInf; s.active = 0; }
        else if (dp <= s.ttol) { s.reason = kConverged; s.active = 0; }
        else if (dp >= 1e5 * s.dp0) { s.reason = kDivergedDtol; s.active = 0; }
        else {
          s.beta = acc_zr[col];
          if (s.beta == 0.0) { s.its += 1; s.reason = kConvergedAtol; s.active = 0; }
          else if (s.beta * s.betaold < 0.0) { s.its += 1; s.reason = kIndefinite; s.active = 0; }
          else if (s.its >= max_it) { s.reason = kDivergedIts; s.active = 0; }
          else s.bfac = s.beta / s.betaold;
        }
      }
      st[col] = s;
    }
    if (dirf) dirf[col] = s.active ? (float)s.bfac : NAN;
    acc_pw[col] = 0.0; acc_zz[col] = 0.0; acc_zr[col] = 0.0;
    act = s.active;
  }
  act = __syncthreads_or(act);
  if (threadIdx.x == 0) dom_active[d] = act;
}

// Step length of every column once p.w is complete (KSPSolve_CG: a = beta / (p.w), 0 for
// columns that stopped or whose curvature changed sign), as floats for the flat update.
__global__ void k_alpha(const ColState* __restrict__ st, const double* __restrict__ acc_pw, float* __restrict__ alphaf,
                        const int* __restrict__ dom_active) {
  const int d = blockIdx.x, lc = threadIdx.x;
  if (lc >= kNLC || (dom_active && !dom_active[d])) return;
  const int64_t col = (int64_t)d * kNLC + lc;
  const ColState s = st[col];
  const double pw = acc_pw[col];
  const bool flip = s.its > 0 && ((pw > 0) != (s.dpi > 0) || pw == 0.0);
  alphaf[col] = (s.active && pw != 0.0 && !flip) ? (float)(s.beta / pw) : 0.f;
}

__global__ void k_count_active(const int* __restrict__ dom_active, int ndom, int* __restrict__ count) {
  __shared__ int sh;
  if (threadIdx.x == 0) sh = 0;
  __syncthreads();
  int c = 0;
  for (int i = threadIdx.x; i < ndom; i += blockDim.x) c += dom_active[i] ? 1 : 0;
  atomicAdd(&sh, c);
  __syncthreads();
  if (threadIdx.x == 0) *count = sh;
}

// -------------------------------------------------------------------------------------
// Mixed precision: outer FP64 residual check, FP64 -> FP32 residual, FP32 correction -> FP64.
__global__ void k_outer_check(ColState* __restrict__ ost, double* __restrict__ acc_zz, double* __restrict__ target,
                              int* __restrict__ dom_active, double rtol, int first) {
  const int d = blockIdx.x, lc = threadIdx.x;
  int act = 0;
  if (lc < kNLC) {
    const int64_t col = (int64_t)d * kNLC + lc;
    ColState s = ost[col];
    const double dp = sqrt(acc_zz[col]);
    if (first) {
      s.dp0 = dp; s.ttol = fmax(rtol * dp, 1e-50); s.its = 0; s.active = 1; s.reason = kIterating;
      s.beta = 0; s.betaold = 0; s.dpi = 0; s.bfac = 0; s.pad = 0;
    }
    s.dp = dp;
    if (s.active) {
      if (!isfinite(dp)) { s.reason = kNanOrInf; s.active = 0; }
      else if (dp <= s.ttol) { s.reason = kConverged; s.active = 0; }
    }
    target[col] = s.active ? 0.5 * s.ttol : 0.0;
    ost[col] = s;
    acc_zz[col] = 0.0;
    act = s.active;
  }
  act = __syncthreads_or(act);
  if (threadIdx.x == 0) dom_active[d] = act;
}

// acc_zz += ||D^-1 r||^2 over interior nodes (FP64 residual norm)
__global__ void __launch_bounds__(kThreads) k_residual_norm(const Tile* __restrict__ tiles,
                                                            const DomDev* __restrict__ doms,
                                                            const uint8_t* __restrict__ flags,
                                                            const double* __restrict__ dinv,
                                                            const double* __restrict__ r, double* __restrict__ acc_zz) {
  __shared__ double red[32];
  const int* dom_active = nullptr;
  DTC_TILE_PROLOGUE
  double zz2 = 0.0;
  if (rowok) {
    for (int i = 0; i < kTileX; ++i) {
      const int xx = t.x0 + i;
      if (xx > D.n[0] - 2) break;
      const int64_t n = node_index(D, xx, yy, zz);
      if (!(flags[n] & kNodeActive)) continue;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double z = dinv[n * 3 + c] * r[vec_index(n, c, lc)];
        zz2 += z * z;
      }
    }
  }
  const double s1 = block_sum_lc<double>(zz2, red);
  if (threadIdx.x < 8) atomicAdd(acc_zz + col, s1);
}

// r32 = (float) (sgn * r64) for columns still refining, 0 otherwise; x32 = p32 = 0 (sgn = -1 when
// r64 holds K X rather than the residual -(K X))
__global__ void __launch_bounds__(kThreads) k_start_inner(const Tile* __restrict__ tiles, const DomDev* __restrict__ doms,
                                                          const uint8_t* __restrict__ flags,
                                                          const double* __restrict__ r64, float* __restrict__ r32,
                                                          float* __restrict__ x32, float* __restrict__ p32,
                                                          const ColState* __restrict__ ost, double sgn) {
  const int* dom_active = nullptr;
  DTC_TILE_PROLOGUE
  if (!rowok) return;
  const bool on = ost[col].active != 0;
  for (int i = 0; i < kTileX; ++i) {
    const int xx = t.x0 + i;
    if (xx > D.n[0] - 2) break;
    const int64_t n = node_index(D, xx, yy, zz);
    if (!(flags[n] & kNodeActive)) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t k = vec_index(n, c, lc);
      r32[k] = on ? (float)(sgn * r64[k]) : 0.0f;
      x32[k] = 0.0f;
      p32[k] = 0.0f;
    }
  }
}

// X += (double) x32 for columns still refining; inner iterations added to the outer count
__global__ void __launch_bounds__(kThreads) k_apply_correction(const Tile* __restrict__ tiles,
                                                               const DomDev* __restrict__ doms,
                                                               const uint8_t* __restrict__ flags,
                                                               const float* __restrict__ x32, double* __restrict__ X,
                                                               const ColState* __restrict__ ost) {
  const int* dom_active = nullptr;
  DTC_TILE_PROLOGUE
  if (!rowok || !ost[col].active) return;
  for (int i = 0; i < kTileX; ++i) {
    const int xx = t.x0 + i;
    if (xx > D.n[0] - 2) break;
    const int64_t n = node_index(D, xx, yy, zz);
    if (!(flags[n] & kNodeActive)) continue;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int64_t k = vec_index(n, c, lc);
      X[k] += (double)x32[k];
    }
  }
}

__global__ void k_add_inner_its(ColState* __restrict__ ost, const ColState* __restrict__ ist, int64_t ncol) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= ncol) return;
  if (ost[i].active) {
    ost[i].its += ist[i].its;
    ost[i].pad += 1;  // refinement steps taken
    if (ist[i].reason == kIndefinite || ist[i].reason == kNanOrInf || ist[i].reason == kDivergedDtol)
      ost[i].betaold = 1.0;  // remembers an inner failure
  }
}

// -------------------------------------------------------------------------------------
// Projection of the reaction forces on the macro shape functions
// (mod_struct_calcmat.f90:246-280): ff((k-1)*NM+l, lc) += F(k, n) * N_l(xi(x_n)), all nodes,
// for the 24 load cases of one column pass; ff is nl x nl per domain (nl = 3 NM) and the
// pass covers columns col0 .. col0+23 (those below nl).
template <int NM>
__global__ void __launch_bounds__(kThreads) k_project(const Tile* __restrict__ tiles, const DomDev* __restrict__ doms,
                                                     const uint8_t* __restrict__ flags, const double* __restrict__ F,
                                                     double* __restrict__ ff, int col0) {
  constexpr int NR = 3 * NM;
  __shared__ double part[4][8][NR + 1];
  const Tile t = tiles[blockIdx.x / 3];
  const DomDev D = doms[t.dom];
  const int lcl = threadIdx.x & 7, lc = (blockIdx.x % 3) * kLcGroup + lcl;
  const int row = threadIdx.x >> 3;
  const int yy = t.y0 + (row & 3), zz = t.z0 + (row >> 2);
  double acc[NR];
#pragma unroll
  for (int k = 0; k < NR; ++k) acc[k] = 0.0;
  if (yy < D.n[1] && zz < D.n[2]) {
    for (int i = 0; i < kTileX; ++i) {
      const int xx = t.x0 + i;
      if (xx >= D.n[0]) break;
      const int64_t n = node_index(D, xx, yy, zz);
      if (!(flags[n] & kNodeActive)) continue;
      double xi[3], N[NM];
      node_xi(D, xx, yy, zz, xi);
      macro_shape_dev<NM>(xi, N);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const double f = F[vec_index(n, k, lc)];
#pragma unroll
        for (int l = 0; l < NM; ++l) acc[k * NM + l] += f * N[l];
      }
    }
  }
  // the 4 rows of a warp that share a load case (lanes lcl, lcl + 8, + 16, + 24), then the warps
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    double v = acc[k];
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    if (lane < 8) part[warp][lane][k] = v;
  }
  __syncthreads();
  const int nl = NR;
  for (int j = threadIdx.x; j < 8 * NR; j += kThreads) {
    const int l8 = j / NR, k = j % NR;
    const double s = part[0][l8][k] + part[1][l8][k] + part[2][l8][k] + part[3][l8][k];
    const int col = col0 + (blockIdx.x % 3) * kLcGroup + l8;
    if (col < nl) atomicAdd(ff + (int64_t)t.dom * nl * nl + k + (int64_t)nl * col, s);
  }
}

// Energy products M(a,b) = u_a . (K u_b) over all nodes, per domain (FP64).  With
// F = K u from the reaction pass, M is the Gram matrix of the load-case solutions in the
// stiffness inner product; ff = vv^-T M equals the reaction projection at the exact solution
// and its error is quadratic in the solution error.  gram is ldg x ldg per domain; X holds the
// load cases row0.. of the block rows, F those of the block columns col0.. (the column passes of
// macro order 2 fill a 72 x 72 Gram block by block).
__global__ void __launch_bounds__(kThreads) k_energy_gram(const Tile* __restrict__ tiles,
                                                          const DomDev* __restrict__ doms,
                                                          const uint8_t* __restrict__ flags,
                                                          const double* __restrict__ X, const double* __restrict__ F,
                                                          double* __restrict__ gram, int ldg, int row0, int col0) {
  __shared__ double part[16][8][25];
  const Tile t = tiles[blockIdx.x / 3];
  const DomDev D = doms[t.dom];
  const int lcl = threadIdx.x & 7, b = (blockIdx.x % 3) * kLcGroup + lcl;
  const int row = threadIdx.x >> 3;
  const int yy = t.y0 + (row & 3), zz = t.z0 + (row >> 2);
  double acc[24];
#pragma unroll
  for (int k = 0; k < 24; ++k) acc[k] = 0.0;
  if (yy < D.n[1] && zz < D.n[2]) {
    for (int i = 0; i < kTileX; ++i) {
      const int xx = t.x0 + i;
      if (xx >= D.n[0]) break;
      const int64_t n = node_index(D, xx, yy, zz);
      if (!(flags[n] & kNodeActive)) continue;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double f = F[vec_index(n, c, b)];
        const double* xu = X + vec_index(n, c, 0);
#pragma unroll
        for (int a = 0; a < 24; ++a) acc[a] += xu[a] * f;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 24; ++k) part[row][lcl][k] = acc[k];
  __syncthreads();
  for (int j = threadIdx.x; j < 8 * 24; j += kThreads) {
    const int l8 = j / 24, a = j % 24;
    double sum = 0.0;
    for (int r2 = 0; r2 < 16; ++r2) sum += part[r2][l8][a];
    const int bg = (blockIdx.x % 3) * kLcGroup + l8;
    atomicAdd(gram + (int64_t)t.dom * ldg * ldg + (row0 + a) + (int64_t)ldg * (col0 + bg), sum);
  }
}

// -------------------------------------------------------------------------------------
// Host driver
struct DeviceSolver::Impl {
  int device = -1;
  cudaStream_t stream = nullptr;
  // persistent buffers grown on demand
  std::vector<std::pair<void**, size_t>> owned;
  void* bufs[80] = {nullptr};
  size_t caps[80] = {0};
  // what the solves of the last batch kept for the adjoint: per chunk the domains (node and
  // voxel offsets of that chunk), their batch positions, and the FP64 displacements, on the
  // device for the chunk solved last (its buffers are still live) or copied to the host
  struct AdjChunk {
    std::vector<DomDev> doms;
    std::vector<int64_t> index;
    int64_t nodes = 0, voxels = 0;
    bool on_device = false;
    std::vector<double> X;       // host checkpoint: nodes * 72
    std::vector<float> svox;     // host checkpoint: voxels
  };
  std::vector<AdjChunk> adj;
  int adj_nen = 0;
  double adj_nu = 0.3;
  bool tensor_matvec = false;   // FP32 inner solve on tcgen05
  bool graphs = true;           // replay CG chunks as CUDA graphs
  // Voxel factors of the next device pass, uploaded while the current one solves: pinned host
  // staging and device slots alternating between passes, copied on their own stream; svox_dev
  // is the slot of the pass being solved (null: the synchronously uploaded bufs[bSvox]).
  cudaStream_t up_stream = nullptr;
  cudaEvent_t up_ev[2] = {nullptr, nullptr};
  float* up_pin[2] = {nullptr, nullptr};
  float* up_dev[2] = {nullptr, nullptr};
  size_t up_cap[2] = {0, 0};
  int up_next = 0;
  float* svox_dev = nullptr;
  float* svox() const { return svox_dev ? svox_dev : static_cast<float*>(bufs[3]); }
  cudaEvent_t ev_solve[2] = {nullptr, nullptr};
  // kernel profiling with CUDA events (opt-in)
  bool profile = false;
  std::vector<cudaEvent_t> ev;
  std::vector<std::pair<int, int>> pending;   // (class, event pair index)
  std::vector<double> dom_mv_bytes, dom_mv_flops, dom_vec_bytes;  // per domain, per launch
  std::vector<int> h_active;                  // domains active at the last chunk boundary
  SolverStats* stats = nullptr;
  int begin(int /*cls*/) {
    if (!profile) return -1;
    const int k = (int)pending.size();
    while ((int)ev.size() < 2 * (k + 1)) { cudaEvent_t e; cudaEventCreate(&e); ev.push_back(e); }
    cudaEventRecord(ev[2 * k], stream);
    return k;
  }
  void end(int cls, int k, double bytes, double flops) {
    if (k < 0) return;
    cudaEventRecord(ev[2 * k + 1], stream);
    pending.push_back({cls, k});
    stats->kc[cls].bytes += bytes;
    stats->kc[cls].flops += flops;
  }
  void flush() {
    if (!profile || pending.empty()) return;
    cudaStreamSynchronize(stream);
    for (auto& pr : pending) {
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[2 * pr.second], ev[2 * pr.second + 1]);
      stats->kc[pr.first].ms += ms;
      stats->kc[pr.first].launches += 1;
    }
    pending.clear();
  }
  // algorithmic traffic of one launch over the domains active at the last chunk boundary
  double active_sum(const std::vector<double>& per_dom) const {
    double t = 0;
    for (size_t d = 0; d < per_dom.size(); ++d) if (h_active.empty() || h_active[d]) t += per_dom[d];
    return t;
  }
};

namespace {

enum Buf { bDoms, bTilesI, bTilesA, bSvox, bFlags, bDinv64, bDinv32, bX, bR64, bP64, bW64, bR32, bX32, bP32, bW32,
           bSt, bOst, bPw, bZz, bZr, bDomAct, bCount, bFf, bTarget, bErr, bBinv32, bBricksI, bBricksA, bZ32, bT32,
           bMgDoms, bMgTiles, bMgSvox, bMgFlags, bMgDinv64, bMgDinv32, bMgBinv32, bMgB, bMgT, bMgZ, bMgMinv, bMgList,
           bAdjG, bAdjV, bAdjBlk, bAdjGrad, bAdjDoms, bAdjX, bAdjSvox, bKe20, bKe20tc, bNodesI, bDirF, bAlphaF,
           bTilesIc, bNodesIc, bBricksIc, bMgTilesC, bMgListC, bCompactCnt, bMgNodes, bMgNodesC, bXkeep, bTilesW,
           bTilesWc, bNumBufs };
static_assert(bNumBufs <= 80, "buffer table");
static_assert(bSvox == 3, "DeviceSolver::Impl::svox() reads bufs[3]");

int ensure(DeviceSolver::Impl& I, int which, size_t bytes, std::string& msg) {
  if (I.caps[which] >= bytes && I.bufs[which]) return DTC_OK;
  if (I.bufs[which]) { cudaFree(I.bufs[which]); I.bufs[which] = nullptr; I.caps[which] = 0; }
  size_t b = std::max<size_t>(bytes, 256);
  DTC_CUDA(cudaMalloc(&I.bufs[which], b));
  I.caps[which] = b;
  return DTC_OK;
}

template <typename T> T* B(DeviceSolver::Impl& I, int which) { return static_cast<T*>(I.bufs[which]); }

int launch_check(std::string& msg) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { msg = std::string("kernel launch: ") + cudaGetErrorString(e); return DTC_ERR_CUDA; }
  return DTC_OK;
}

}  // namespace

DeviceSolver::DeviceSolver() : impl_(new Impl) {}
DeviceSolver::~DeviceSolver() {
  if (impl_) {
    if (impl_->device >= 0) cudaSetDevice(impl_->device);
    for (cudaEvent_t e : impl_->ev) cudaEventDestroy(e);
    for (cudaEvent_t e : impl_->ev_solve) if (e) cudaEventDestroy(e);
    for (void* b : impl_->bufs) if (b) cudaFree(b);
    for (int k = 0; k < 2; ++k) {
      if (impl_->up_ev[k]) cudaEventSynchronize(impl_->up_ev[k]);
      if (impl_->up_pin[k]) cudaFreeHost(impl_->up_pin[k]);
      if (impl_->up_dev[k]) cudaFree(impl_->up_dev[k]);
      if (impl_->up_ev[k]) cudaEventDestroy(impl_->up_ev[k]);
    }
    if (impl_->up_stream) cudaStreamDestroy(impl_->up_stream);
    if (impl_->stream) cudaStreamDestroy(impl_->stream);
    delete impl_;
  }
}

int DeviceSolver::init(int device, std::string& msg) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { msg = "no CUDA device"; return DTC_ERR_NO_DEVICE; }
  if (device < 0 || device >= n) { msg = "device ordinal out of range"; return DTC_ERR_INVALID_ARGUMENT; }
  DTC_CUDA(cudaSetDevice(device));
  DTC_CUDA(cudaStreamCreateWithFlags(&impl_->stream, cudaStreamNonBlocking));
  impl_->device = device;
  return DTC_OK;
}

void launch_sweep_tc(int mode, const Tile* tiles, int64_t ntiles, const DomDev* doms, const float* svox,
                     const uint8_t* flags, const float* binv, const float* b, const float* u, float* y, float scale,
                     float omega, double* acc1, double* acc2, const int* dom_active, int* err, cudaStream_t s);
int allow_sweep_tc(std::string& msg);
int upload_tc_operand(const double* khat, cudaStream_t s, std::string& msg);
int set_tc_spin_limit(long long spins, cudaStream_t s, std::string& msg);
void build_tc20_operand(const double* k20, float* img);
size_t tc20_operand_bytes();
int allow_ebe_tc(std::string& msg);
void launch_ebe_tc(const Tile* bricks, int64_t nb, const DomDev* doms, const float* svox, const uint8_t* flags,
                   const float* bsplit, const float* u, float* y, double scale, double* acc_pw, const int* dom_active,
                   int* err, cudaStream_t s);

namespace {

// CG on one precision: x (interior part), r = b on entry, p = 0 on entry.
template <typename T, int NEN, bool ALL, bool DOT>
void launch_ebe(const Tile* bricks, int64_t nb, const DomDev* dd, const float* svox, const uint8_t* fl, const T* ke,
                const T* u, T* y, double scale, double* acc, const int* act, cudaStream_t s) {
  using S = EbeShape<T, NEN>;
  if (nb <= 0) return;
  k_ebe<T, NEN, ALL, DOT><<<(unsigned)(S::NGRP * nb), S::kThreadsEbe, S::smem, s>>>(bricks, dd, svox, fl, ke, u, y,
                                                                                    scale, acc, act);
}

template <typename T, int NEN, bool ALL, bool DOT>
int allow_ebe_smem(std::string& msg) {
  DTC_CUDA(cudaFuncSetAttribute(k_ebe<T, NEN, ALL, DOT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)EbeShape<T, NEN>::smem));
  return DTC_OK;
}

template <int NEN>
int allow_all_ebe(std::string& msg) {
  int e;
  if ((e = allow_ebe_smem<float, NEN, false, true>(msg))) return e;
  if ((e = allow_ebe_smem<float, NEN, false, false>(msg))) return e;   // multigrid residual sweeps
  if ((e = allow_ebe_smem<double, NEN, false, true>(msg))) return e;
  if ((e = allow_ebe_smem<double, NEN, false, false>(msg))) return e;
  if ((e = allow_ebe_smem<double, NEN, true, false>(msg))) return e;
  return DTC_OK;
}

// Work lists of one solve: node tiles (vector kernels and the HEX08 node-centric operator)
// and voxel bricks (HEX20 element-by-element operator), over the interior / all nodes.
struct Work {
  const Tile *ti, *ta, *bi, *ba;
  int64_t nti, nta, nbi, nba;
  const int64_t* nodes;  // active interior nodes, (domain << kListShift) | node
  int64_t nnodes;
  const double* ke64;   // HEX20 unit element matrix (FP64, then its FP32 copy)
  const float* ke32;
  const float* ke20tc;  // HEX20 FP32 applications on tcgen05: split matrix in the B layout, else null
  int* err;             // mbarrier time-out flag of the tensor-core kernels
  int minb32 = 6;       // HEX08 slab sweeps: CTAs per SM of the FP32 CG application (6 or 8)
  int minb64 = 4;       //                    and of every FP64 application (4 or 6)
  const Tile* tw = nullptr;   // interior sweep tiles (rows of kSweepX nodes) of the slab sweeps
  int64_t ntw = 0;
};

// y = scale * K u on the interior (ALL = false) or every node; DOT: acc[col] += u . y.
template <typename T, int NEN, bool ALL, bool DOT>
void apply_k(const Work& W, const DomDev* dd, const float* svox, const uint8_t* fl, const T* u, T* y, double scale,
             double* acc, const int* act, cudaStream_t s, int bnd_only = 0) {
  if constexpr (NEN == 8) {
    // interior: the sweep tiles (rows of kSweepX nodes); every node: the node tiles
    const int64_t nt = ALL ? W.nta : W.ntw;
    if (nt <= 0) return;
    const unsigned g = (unsigned)(3 * nt);
    const Tile* tl = ALL ? W.ta : W.tw;
    const int xl = ALL ? kTileX : kSweepX;
    if constexpr (sizeof(T) == 4) {
      if (W.minb32 == 8) k_matvec<T, ALL, DOT, 8><<<g, kThreads, 0, s>>>(tl, dd, svox, u, y, scale, acc, act, bnd_only, xl);
      else k_matvec<T, ALL, DOT, 6><<<g, kThreads, 0, s>>>(tl, dd, svox, u, y, scale, acc, act, bnd_only, xl);
    } else {
      if (W.minb64 == 6) k_matvec<T, ALL, DOT, 6><<<g, kThreads, 0, s>>>(tl, dd, svox, u, y, scale, acc, act, bnd_only, xl);
      else k_matvec<T, ALL, DOT, 4><<<g, kThreads, 0, s>>>(tl, dd, svox, u, y, scale, acc, act, bnd_only, xl);
    }
  } else {
    const T* ke;
    if constexpr (sizeof(T) == 8) ke = W.ke64;
    else ke = W.ke32;
    if constexpr (sizeof(T) == 4 && !ALL) {
      if (W.ke20tc) {
        launch_ebe_tc(W.bi, W.nbi, dd, svox, fl, W.ke20tc, u, y, scale, DOT ? acc : nullptr, act, W.err, s);
        return;
      }
    }
    launch_ebe<T, NEN, ALL, DOT>(ALL ? W.ba : W.bi, ALL ? W.nba : W.nbi, dd, svox, fl, ke, u, y, scale, acc, act, s);
  }
}


// -------------------------------------------------------------------------------------
// Multigrid hierarchy of one solve (HEX08, FP32 inner solve).  Level 0 is the fine grid
// already packed; levels >= 1 live in their own node / voxel arrays.  Per level: DomDev for
// every domain (L = 0 where the domain has no such level), interior tiles of the domains that
// smooth on the level (sm), interior tiles of every domain present (in: restriction target),
// all tiles (node set-up), and the domains whose coarsest level it is (dense solve).
struct MgPlan {
  int nlev = 0;
  float omega = 0.f;                                // damping on the HEX08 levels
  float omega0 = 0.f;                               // damping on the fine level (HEX08 or HEX20)
  std::vector<DomDev> doms;                         // nlev * ndom, level-major
  std::vector<Tile> tiles;
  std::vector<int64_t> sm_off, sm_n, in_off, in_n, all_off, all_n;
  std::vector<int64_t> sw_off, sw_n;                // smoothing tiles as rows of kSweepX nodes (slab sweeps)
  std::vector<int> lists;
  std::vector<int64_t> list_off, list_n;
  std::vector<int64_t> nodes_l;                     // levels >= 1: active interior nodes, (domain << kListShift) | node
  std::vector<int64_t> nl_off, nl_n;
  std::vector<float> svox;                          // voxels of levels >= 1
  std::vector<float> minv;                          // ndom * 81 * 81
  int64_t nodes = 0;                                // nodes of levels >= 1
};

// Largest eigenvalue of Khat v = lambda De v, De the node-block (3x3) diagonal of the unit
// voxel matrix: bounds lambda_max(D^-1 K) of every assembly of scaled voxels, D its node-block
// diagonal (x^T K x = sum_v x_v^T K_v x_v <= lambda sum_v x_v^T De_v x_v = lambda x^T D x).
double block_jacobi_bound(const double* kh, int nen) {
  const int nd = 3 * nen;
  std::vector<double> inv((size_t)nen * 9), v(nd), w(nd), kv(nd);
  for (int a = 0; a < nen; ++a) {
    double m[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) m[3 * i + j] = kh[(3 * a + i) + nd * (3 * a + j)];
    const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[2] * m[7] - m[1] * m[8], c02 = m[1] * m[5] - m[2] * m[4];
    const double det = m[0] * c00 + m[3] * c01 + m[6] * c02;
    double* q = &inv[(size_t)a * 9];
    q[0] = c00 / det; q[1] = c01 / det; q[2] = c02 / det;
    q[3] = (m[5] * m[6] - m[3] * m[8]) / det; q[4] = (m[0] * m[8] - m[2] * m[6]) / det;
    q[5] = (m[2] * m[3] - m[0] * m[5]) / det;
    q[6] = (m[3] * m[7] - m[4] * m[6]) / det; q[7] = (m[1] * m[6] - m[0] * m[7]) / det;
    q[8] = (m[0] * m[4] - m[1] * m[3]) / det;
  }
  double lam = 0;
  for (int i = 0; i < nd; ++i) v[i] = 1.0 + 0.01 * i;
  for (int it = 0; it < 3000; ++it) {
    for (int i = 0; i < nd; ++i) {
      double s = 0;
      for (int j = 0; j < nd; ++j) s += kh[i + nd * j] * v[j];
      kv[i] = s;
    }
    double vkv = 0, vdv = 0;
    for (int a = 0; a < nen; ++a)
      for (int i = 0; i < 3; ++i) {
        double dv = 0;
        for (int j = 0; j < 3; ++j) dv += kh[(3 * a + i) + nd * (3 * a + j)] * v[3 * a + j];
        vdv += v[3 * a + i] * dv;
        vkv += v[3 * a + i] * kv[3 * a + i];
      }
    lam = vkv / vdv;
    double nrm = 0;
    for (int a = 0; a < nen; ++a)
      for (int i = 0; i < 3; ++i) {
        double s = 0;
        for (int j = 0; j < 3; ++j) s += inv[(size_t)a * 9 + 3 * i + j] * kv[3 * a + j];
        w[3 * a + i] = s;
        nrm += s * s;
      }
    nrm = std::sqrt(nrm);
    for (int i = 0; i < nd; ++i) v[i] = w[i] / nrm;
  }
  return lam;
}

// Dense inverse of the coarsest operator over its <= 27 interior nodes (FP64 Cholesky; pivots
// below 1e-12 of the largest diagonal entry are dropped, so floating pieces without a fixed
// node get a zero correction), stored as float 81 x 81.
void coarse_inverse(const DomDev& D, const float* sv, const double* kh, float* out) {
  constexpr int N = kMgDenseN;
  double A[N * N];
  std::memset(A, 0, sizeof(A));
  const int ix = D.n[0] - 2, iy = D.n[1] - 2, iz = D.n[2] - 2;
  auto dof = [&](int x, int y, int z, int c) -> int {
    if (x < 1 || y < 1 || z < 1 || x > ix || y > iy || z > iz) return -1;
    return 3 * ((x - 1) + 3 * (y - 1) + 9 * (z - 1)) + c;
  };
  for (int vz = 0; vz < D.L[2]; ++vz)
    for (int vy = 0; vy < D.L[1]; ++vy)
      for (int vx = 0; vx < D.L[0]; ++vx) {
        const double s = (double)sv[vx + D.L[0] * (vy + D.L[1] * vz)] * D.scale;
        if (s == 0.0) continue;
        for (int a = 0; a < 8; ++a)
          for (int ca = 0; ca < 3; ++ca) {
            const int ra = dof(vx + Elem<8>::off(a, 0), vy + Elem<8>::off(a, 1), vz + Elem<8>::off(a, 2), ca);
            if (ra < 0) continue;
            for (int b = 0; b < 8; ++b)
              for (int cb = 0; cb < 3; ++cb) {
                const int rb = dof(vx + Elem<8>::off(b, 0), vy + Elem<8>::off(b, 1), vz + Elem<8>::off(b, 2), cb);
                if (rb < 0) continue;
                A[ra * N + rb] += s * kh[(3 * a + ca) + 24 * (3 * b + cb)];
              }
          }
      }
  double dmax = 0;
  for (int i = 0; i < N; ++i) dmax = std::max(dmax, A[i * N + i]);
  bool keep[N];
  double Lc[N * N];
  std::memset(Lc, 0, sizeof(Lc));
  for (int j = 0; j < N; ++j) {
    double d = A[j * N + j];
    for (int k = 0; k < j; ++k) d -= Lc[j * N + k] * Lc[j * N + k];
    keep[j] = dmax > 0 && d > 1e-12 * dmax;
    if (!keep[j]) continue;
    const double ljj = std::sqrt(d);
    Lc[j * N + j] = ljj;
    for (int i = j + 1; i < N; ++i) {
      double s = A[i * N + j];
      for (int k = 0; k < j; ++k) s -= Lc[i * N + k] * Lc[j * N + k];
      Lc[i * N + j] = s / ljj;
    }
  }
  // A^-1 = L^-T L^-1 on the kept DOFs: the lower-triangular inverse column by column, then the
  // symmetric product (rows and columns of dropped DOFs are zero)
  double Li[N * N];
  std::memset(Li, 0, sizeof(Li));
  for (int j = 0; j < N; ++j) {
    if (!keep[j]) continue;
    Li[j * N + j] = 1.0 / Lc[j * N + j];
    for (int i = j + 1; i < N; ++i) {
      if (!keep[i]) continue;
      double s = 0.0;
      for (int k = j; k < i; ++k) s -= Lc[i * N + k] * Li[k * N + j];
      Li[i * N + j] = s / Lc[i * N + i];
    }
  }
  for (int i = 0; i < N; ++i)
    for (int c = 0; c <= i; ++c) {
      double s = 0.0;
      for (int k = i; k < N; ++k) s += Li[k * N + i] * Li[k * N + c];
      out[i * N + c] = out[c * N + i] = (float)s;
    }
}

// Build the hierarchy on the host from the fine voxel factors.  fine_i / fine_w: interior node
// tiles / sweep tiles of the fine level (level-0 smoothing tiles are those of domains with a
// coarser level).
// Levels from this one down smooth twice per visit (pre and post): on 256 x 32^3 and on an
// uneven batch (16^3-64^3) ~3.5% less solve time than once everywhere; twice already on
// level 1 costs more than the iterations it saves.
constexpr int kMgTwiceFrom = 2;

// HEX20 fine grids (m = 2) get one p-coarsening first: level 1 is the HEX08 mesh of the same
// voxels (corner nodes; the trilinear space is contained in the serendipity one, so the
// exactly integrated HEX08 matrix is the Galerkin product of the HEX20 one), then the voxel
// grids are halved as for HEX08.  Every domain's levels are built on their own host thread,
// then concatenated in domain order (the layout does not depend on the thread count).
void build_mg(MgPlan& P, const std::vector<DomDev>& doms0, const std::vector<float>& svox0,
              const std::vector<Tile>& fine_i, const std::vector<Tile>& fine_w, double nu, int nen, int threads) {
  const int ndom = (int)doms0.size();
  double kh[576];
  voxel_stiffness(8, nu, kh);
  auto step = [](double lam) { return (float)(1.0 / (0.5 * (1.1 + 1.0 / 30.0) * lam)); };
  P.omega = step(block_jacobi_bound(kh, 8));
  if (nen == 20) {
    std::vector<double> k20(3600);
    voxel_stiffness(20, nu, k20.data());
    P.omega0 = step(block_jacobi_bound(k20.data(), 20));
  } else {
    P.omega0 = P.omega;
  }
  std::vector<int> nlev(ndom, 1);
  int nl = 1;
  for (int d = 0; d < ndom; ++d) {
    int L[3] = {doms0[d].L[0], doms0[d].L[1], doms0[d].L[2]};
    if (doms0[d].m == 2) ++nlev[d];   // the HEX08 level of the same voxels
    while (std::max(L[0], std::max(L[1], L[2])) > kMgMaxCoarse) {
      for (int k = 0; k < 3; ++k) L[k] = (L[k] + 1) / 2;
      ++nlev[d];
    }
    nl = std::max(nl, nlev[d]);
  }
  // per domain and level >= 1: grid, voxel factors, work lists (offsets filled in later)
  struct Level {
    DomDev C;
    std::vector<float> sv;
    std::vector<Tile> t_in, t_sm, t_all, t_sw;
    std::vector<int32_t> n_in;   // active interior nodes (index inside the level's grid)
  };
  std::vector<std::vector<Level>> lev(ndom);
  P.minv.assign((size_t)ndom * kMgDenseN * kMgDenseN, 0.f);
  parallel_for(ndom, threads, [&](int64_t dd) {
    const int d = (int)dd;
    std::vector<float> cur(svox0.begin() + doms0[d].vox_off,
                           svox0.begin() + doms0[d].vox_off + (int64_t)doms0[d].L[0] * doms0[d].L[1] * doms0[d].L[2]);
    DomDev F = doms0[d];
    lev[d].resize(nlev[d]);
    for (int l = 1; l < nlev[d]; ++l) {
      Level& Lv = lev[d][l];
      DomDev C = F;
      const bool pc = F.m == 2;   // p-coarsening: same voxels, corner nodes
      for (int k = 0; k < 3; ++k) { C.L[k] = pc ? F.L[k] : (F.L[k] + 1) / 2; C.n[k] = C.L[k] + 1; }
      C.m = 1;
      C.scale = pc ? F.scale : 2.0 * F.scale;
      std::vector<float> nv((size_t)C.L[0] * C.L[1] * C.L[2], 0.f);
      if (pc) {
        nv = cur;
      } else {
        for (int z = 0; z < F.L[2]; ++z)
          for (int y = 0; y < F.L[1]; ++y)
            for (int x = 0; x < F.L[0]; ++x)
              nv[(x / 2) + (size_t)C.L[0] * ((y / 2) + (size_t)C.L[1] * (z / 2))] +=
                  0.125f * cur[x + (size_t)F.L[0] * (y + (size_t)F.L[1] * z)];
      }
      // activity and tiles
      const int nx = C.n[0], ny = C.n[1], nz = C.n[2];
      std::vector<uint8_t> act((size_t)nx * ny * nz, 0);
      for (int z = 0; z < C.L[2]; ++z)
        for (int y = 0; y < C.L[1]; ++y)
          for (int x = 0; x < C.L[0]; ++x) {
            if (nv[x + (size_t)C.L[0] * (y + (size_t)C.L[1] * z)] == 0.f) continue;
            for (int c = 0; c < 2; ++c)
              for (int b = 0; b < 2; ++b)
                for (int a = 0; a < 2; ++a) act[(x + a) + (size_t)nx * ((y + b) + (size_t)ny * (z + c))] = 1;
          }
      auto any = [&](int x0, int y0, int z0, int lo, int hx, int hy, int hz, int sx = kTileX) {
        for (int z = std::max(z0, lo); z < std::min(z0 + kTileZ, hz + 1); ++z)
          for (int y = std::max(y0, lo); y < std::min(y0 + kTileY, hy + 1); ++y)
            for (int x = std::max(x0, lo); x < std::min(x0 + sx, hx + 1); ++x)
              if (act[x + (size_t)nx * (y + (size_t)ny * z)]) return true;
        return false;
      };
      for (int z0 = 1; z0 <= nz - 2; z0 += kTileZ)
        for (int y0 = 1; y0 <= ny - 2; y0 += kTileY)
          for (int x0 = 1; x0 <= nx - 2; x0 += kTileX)
            if (any(x0, y0, z0, 1, nx - 2, ny - 2, nz - 2)) {
              const Tile t{d, (int16_t)x0, (int16_t)y0, (int16_t)z0, 0};
              Lv.t_in.push_back(t);
              if (nlev[d] > l + 1) Lv.t_sm.push_back(t);
            }
      for (int z0 = 0; z0 <= nz - 1; z0 += kTileZ)
        for (int y0 = 0; y0 <= ny - 1; y0 += kTileY)
          for (int x0 = 0; x0 <= nx - 1; x0 += kTileX)
            if (any(x0, y0, z0, 0, nx - 1, ny - 1, nz - 1))
              Lv.t_all.push_back(Tile{d, (int16_t)x0, (int16_t)y0, (int16_t)z0, 0});
      if (nlev[d] > l + 1)
        for (int z0 = 1; z0 <= nz - 2; z0 += kTileZ)
          for (int y0 = 1; y0 <= ny - 2; y0 += kTileY)
            for (int x0 = 1; x0 <= nx - 2; x0 += kSweepX)
              if (any(x0, y0, z0, 1, nx - 2, ny - 2, nz - 2, kSweepX))
                Lv.t_sw.push_back(Tile{d, (int16_t)x0, (int16_t)y0, (int16_t)z0, 0});
      for (int z = 1; z < nz - 1; ++z)
        for (int y = 1; y < ny - 1; ++y)
          for (int x = 1; x < nx - 1; ++x) {
            const int32_t k = x + nx * (y + ny * z);
            if (act[k]) Lv.n_in.push_back(k);
          }
      Lv.C = C;
      Lv.sv = nv;
      cur.swap(nv);
      F = C;
    }
    // coarsest level: dense inverse (its grid is lev[d].back().C, or the fine one)
    const DomDev& Cc = nlev[d] > 1 ? lev[d][nlev[d] - 1].C : doms0[d];
    coarse_inverse(Cc, cur.data(), kh, &P.minv[(size_t)d * kMgDenseN * kMgDenseN]);
  });
  // concatenate in domain order
  P.nlev = nl;
  P.doms.assign((size_t)nl * ndom, DomDev{});
  P.sm_off.assign(nl, 0); P.sm_n.assign(nl, 0); P.in_off.assign(nl, 0); P.in_n.assign(nl, 0);
  P.sw_off.assign(nl, 0); P.sw_n.assign(nl, 0);
  P.all_off.assign(nl, 0); P.all_n.assign(nl, 0); P.list_off.assign(nl, 0); P.list_n.assign(nl, 0);
  P.nl_off.assign(nl, 0); P.nl_n.assign(nl, 0);
  P.tiles.clear(); P.lists.clear(); P.svox.clear(); P.nodes_l.clear(); P.nodes = 0;
  for (int d = 0; d < ndom; ++d) P.doms[d] = doms0[d];
  P.sm_off[0] = 0;
  for (const Tile& t : fine_i) if (nlev[t.dom] > 1) P.tiles.push_back(t);
  P.sm_n[0] = (int64_t)P.tiles.size();
  P.sw_off[0] = (int64_t)P.tiles.size();
  for (const Tile& t : fine_w) if (nlev[t.dom] > 1) P.tiles.push_back(t);
  P.sw_n[0] = (int64_t)P.tiles.size() - P.sw_off[0];
  for (int l = 1; l < nl; ++l) {
    for (int d = 0; d < ndom; ++d) {
      if (nlev[d] <= l) continue;
      Level& Lv = lev[d][l];
      Lv.C.vox_off = (int64_t)P.svox.size();
      Lv.C.node_off = P.nodes;
      P.svox.insert(P.svox.end(), Lv.sv.begin(), Lv.sv.end());
      P.nodes += (int64_t)Lv.C.n[0] * Lv.C.n[1] * Lv.C.n[2];
      P.doms[(size_t)l * ndom + d] = Lv.C;
    }
    auto append = [&](std::vector<Tile> Level::*member, int64_t& off, int64_t& cnt) {
      off = (int64_t)P.tiles.size();
      for (int d = 0; d < ndom; ++d)
        if (nlev[d] > l) P.tiles.insert(P.tiles.end(), (lev[d][l].*member).begin(), (lev[d][l].*member).end());
      cnt = (int64_t)P.tiles.size() - off;
    };
    append(&Level::t_sm, P.sm_off[l], P.sm_n[l]);
    append(&Level::t_in, P.in_off[l], P.in_n[l]);
    append(&Level::t_all, P.all_off[l], P.all_n[l]);
    append(&Level::t_sw, P.sw_off[l], P.sw_n[l]);
    P.nl_off[l] = (int64_t)P.nodes_l.size();
    for (int d = 0; d < ndom; ++d)
      if (nlev[d] > l)
        for (const int32_t k : lev[d][l].n_in)
          P.nodes_l.push_back(((int64_t)d << kListShift) | (lev[d][l].C.node_off + k));
    P.nl_n[l] = (int64_t)P.nodes_l.size() - P.nl_off[l];
  }
  for (int l = 0; l < nl; ++l) {
    P.list_off[l] = (int64_t)P.lists.size();
    for (int d = 0; d < ndom; ++d)
      if (nlev[d] - 1 == l) P.lists.push_back(d);
    P.list_n[l] = (int64_t)P.lists.size() - P.list_off[l];
  }
}

// One V-cycle z_0 = B r_0 for every active domain; on level 0 accumulates z.z and z.r.
struct MgDev {
  const MgPlan* P;
  int ndom;
  const Tile* tiles;
  const DomDev* doms0;   // fine level
  const DomDev* doms;    // nlev * ndom
  const float *svox0, *svox, *binv0, *binv, *minv;
  const uint8_t *flags0, *flags;
  const int* lists;
  const int64_t* nodes;  // levels >= 1: active interior nodes (segments nl_off / nl_n of the plan)
  float *b, *t, *z;      // levels >= 1
  float *t0, *z0;        // fine level
  int nen0;              // element of the fine level; HEX20 applies K with the brick kernel
  const Tile* bricks0;   // fine-level interior bricks (HEX20)
  int64_t nbricks0;
  const int64_t* nodes0; // fine-level active interior nodes, (domain << kListShift) | node
  int64_t nnodes0;
  const float* ke32;     // HEX20 unit element matrix (FP32)
  const float* ke20tc;   // its tensor-core operand, or null (brick SIMT kernel)
  int* err;
  int minb_res = 6, minb_post = 6;   // HEX08 residual / post-smoothing sweeps: CTAs per SM (6 or 8)
};

// The HEX08 residual and post-smoothing sweeps with the tuned register budget (the fine
// level's choice, used on the coarse levels too).
// t: sweep tiles (rows of kSweepX nodes), g = 3 x their number.
template <int MODE, bool DOT>
void launch_mg_matvec(int minb, unsigned g, cudaStream_t s, const Tile* t, const DomDev* d, const float* sv,
                      const float* bi, const float* b, const float* u, float* y, float om, double* a1, double* a2,
                      const int* act) {
  if (g == 0) return;
  if (minb == 8) k_mg_matvec<MODE, DOT, 8><<<g, kThreads, 0, s>>>(t, d, sv, bi, b, u, y, om, a1, a2, act, kSweepX);
  else k_mg_matvec<MODE, DOT, 6><<<g, kThreads, 0, s>>>(t, d, sv, bi, b, u, y, om, a1, a2, act, kSweepX);
}

// t_ready: the fine-level t = omega D^-1 r0 was already written (by k_update_flat)
void mg_vcycle(DeviceSolver::Impl& I, const MgDev& M, int l, const float* r0, double* zz, double* zr, const int* act,
               int64_t& launches, bool t_ready = false) {
  cudaStream_t s = I.stream;
  const MgPlan& P = *M.P;
  const DomDev* dl = l == 0 ? M.doms0 : M.doms + (size_t)l * M.ndom;
  const float* sv = l == 0 ? M.svox0 : M.svox;
  const float* bi = l == 0 ? M.binv0 : M.binv;
  const uint8_t* fl = l == 0 ? M.flags0 : M.flags;
  const float* b = l == 0 ? r0 : M.b;
  float* t = l == 0 ? M.t0 : M.t;
  float* z = l == 0 ? M.z0 : M.z;
  // fine-level launches are profiled one by one with their algorithmic work; the coarser
  // levels as one class
  const bool fine = l == 0;
  const double vb = I.profile && fine ? I.active_sum(I.dom_vec_bytes) * sizeof(float) : 0;
  const double mb = I.profile && fine ? I.active_sum(I.dom_mv_bytes) * sizeof(float) : 0;
  const double mf = I.profile && fine ? I.active_sum(I.dom_mv_flops) : 0;
  const int q0 = fine ? -1 : I.begin(0);
  if (P.list_n[l] > 0) {
    if (l == 0)
      k_mg_coarse<true><<<(unsigned)P.list_n[l], 256, 0, s>>>(M.lists + P.list_off[l], dl, M.minv, b, z, zz, zr, act);
    else
      k_mg_coarse<false><<<(unsigned)P.list_n[l], 256, 0, s>>>(M.lists + P.list_off[l], dl, M.minv, b, z, nullptr,
                                                               nullptr, act);
    ++launches;
  }
  const int64_t nsm = P.sm_n[l];
  if (nsm == 0 || l + 1 >= P.nlev) {
    if (!fine) I.end(kcMgCoarse, q0, 0, 0);
    return;
  }
  const Tile* tsm = M.tiles + P.sm_off[l];
  const unsigned g = (unsigned)(3 * nsm);
  const Tile* tsw = M.tiles + P.sw_off[l];        // the slab sweeps' rows of kSweepX nodes
  const unsigned gw = (unsigned)(3 * P.sw_n[l]);
  int q = -1;
  if (!(fine && t_ready)) {
    q = fine ? I.begin(0) : -1;
    const int64_t items = (int64_t)kQuads * (fine ? M.nnodes0 : P.nl_n[l]);
    if (items > 0)
      k_mg_jacobi_flat<<<(unsigned)((items + 255) / 256), 256, 0, s>>>(fine ? M.nodes0 : M.nodes + P.nl_off[l], items,
                                                                         M.doms + (size_t)(l + 1) * M.ndom, bi, b,
                                                                         fine ? P.omega0 : P.omega, t, act);
    if (fine) I.end(kcMgJacobi, q, 2 * vb + vb / 12, 0);   // b in, t out, 6 floats of D^-1 per node
    ++launches;
  }
  q = fine ? I.begin(0) : -1;
  const float om = fine ? P.omega0 : P.omega;
  // deeper levels smooth twice before and after their coarse correction (their grids are small)
  const bool twice = !fine && l >= kMgTwiceFrom;
  float* cur = t;                  // the smoothed iterate
  float* rbuf = z;                 // the residual handed to the restriction
  if (twice) {
    launch_mg_matvec<kMgPost, false>(M.minb_post, gw, s, tsw, dl, sv, bi, b, t, z, om, nullptr, nullptr, act);
    ++launches;
    cur = z;
    rbuf = t;
  }
  if (fine && M.nen0 == 20) {
    if (M.ke20tc)
      launch_ebe_tc(M.bricks0, M.nbricks0, dl, sv, fl, M.ke20tc, t, z, -1.0, nullptr, act, M.err, s);
    else
      launch_ebe<float, 20, false, false>(M.bricks0, M.nbricks0, dl, sv, fl, M.ke32, t, z, -1.0, nullptr, act, s);
    k_mg_combine<kMgRes, false><<<g, kThreads, 0, s>>>(tsm, dl, fl, bi, b, t, z, om, nullptr, nullptr, act);
    ++launches;
  } else if (fine && I.tensor_matvec) {
    launch_sweep_tc(kTcRes, tsm, nsm, dl, sv, fl, bi, b, cur, rbuf, 1.0f, om, nullptr, nullptr, act, M.err, s);
  } else if (fine) {
    launch_mg_matvec<kMgRes, false>(M.minb_res, gw, s, tsw, dl, sv, bi, b, cur, rbuf, om, nullptr, nullptr, act);
  } else {
    launch_mg_matvec<kMgRes, false>(M.minb_res, gw, s, tsw, dl, sv, bi, b, cur, rbuf, om, nullptr, nullptr, act);
  }
  if (fine) I.end(kcMgResidual, q, mb + vb, mf);          // t in, r out (mb), b in
  const DomDev* dc = M.doms + (size_t)(l + 1) * M.ndom;
  q = fine ? I.begin(0) : -1;
  {
    const int64_t items = (int64_t)kQuads * P.nl_n[l + 1];
    if (items > 0)
      k_mg_restrict_flat<<<(unsigned)((items + 255) / 256), 256, 0, s>>>(M.nodes + P.nl_off[l + 1], items, dc, dl,
                                                                           rbuf, M.b, act);
  }
  if (fine) I.end(kcMgTransfer, q, vb * (1.0 + 1.0 / 8.0), 0);
  launches += 2;
  if (!fine) I.end(kcMgCoarse, q0, 0, 0);
  mg_vcycle(I, M, l + 1, r0, zz, zr, act, launches);
  const int q1 = fine ? -1 : I.begin(0);
  q = fine ? I.begin(0) : -1;
  {
    const int64_t items = (int64_t)kQuads * (fine ? M.nnodes0 : P.nl_n[l]);
    if (items > 0)
      k_mg_prolong_flat<<<(unsigned)((items + 255) / 256), 256, 0, s>>>(fine ? M.nodes0 : M.nodes + P.nl_off[l],
                                                                          items, dl, dc, M.z, cur, act);
  }
  if (fine) I.end(kcMgTransfer, q, vb * (2.0 + 1.0 / 8.0), 0);
  q = fine ? I.begin(0) : -1;
  if (l == 0 && M.nen0 == 20) {
    if (M.ke20tc)
      launch_ebe_tc(M.bricks0, M.nbricks0, dl, sv, fl, M.ke20tc, t, z, -1.0, nullptr, act, M.err, s);
    else
      launch_ebe<float, 20, false, false>(M.bricks0, M.nbricks0, dl, sv, fl, M.ke32, t, z, -1.0, nullptr, act, s);
    k_mg_combine<kMgPost, true><<<g, kThreads, 0, s>>>(tsm, dl, fl, bi, b, t, z, P.omega0, zz, zr, act);
    ++launches;
  } else if (l == 0 && I.tensor_matvec)
    launch_sweep_tc(kTcPost, tsm, nsm, dl, sv, fl, bi, b, t, z, 1.0f, P.omega0, zz, zr, act, M.err, s);
  else if (l == 0)
    launch_mg_matvec<kMgPost, true>(M.minb_post, gw, s, tsw, dl, sv, bi, b, t, z, P.omega0, zz, zr, act);
  else if (twice) {
    // z holds the corrected iterate: t = z + w D^-1 (b - K z), then z = t + w D^-1 (b - K t)
    launch_mg_matvec<kMgPost, false>(M.minb_post, gw, s, tsw, dl, sv, bi, b, z, t, P.omega, nullptr, nullptr, act);
    launch_mg_matvec<kMgPost, false>(M.minb_post, gw, s, tsw, dl, sv, bi, b, t, z, P.omega, nullptr, nullptr, act);
    ++launches;
  } else
    launch_mg_matvec<kMgPost, false>(M.minb_post, gw, s, tsw, dl, sv, bi, b, t, z, P.omega, nullptr, nullptr, act);
  if (fine) I.end(kcMgPost, q, mb + vb + vb / 12, mf);     // t in, z out (mb), b in, D^-1
  if (!fine) I.end(kcMgCoarse, q1, 0, 0);
  launches += 2;
}

// One chunk of CG iterations replayed as a CUDA graph: captured on first use (every kernel
// argument is fixed for the whole solve), then one cudaGraphLaunch per chunk instead of a few
// hundred launches.  Profiling runs launch directly so that their event records stay per kernel.
struct ChunkGraph {
  cudaGraphExec_t exec = nullptr;
  int64_t launches = 0;   // kernels in one chunk
  ~ChunkGraph() { reset(); }
  void reset() {   // the next run captures again (the work lists changed)
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
  }
  template <class Body>
  int run(cudaStream_t s, bool direct, int64_t& counter, Body&& body, std::string& msg) {
    if (direct) {
      body(counter);
      return DTC_OK;
    }
    if (!exec) {
      cudaGraph_t g = nullptr;
      DTC_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      int64_t n = 0;
      body(n);
      const cudaError_t ec = cudaStreamEndCapture(s, &g);
      if (ec != cudaSuccess) { msg = std::string("chunk capture: ") + cudaGetErrorString(ec); return DTC_ERR_CUDA; }
      const cudaError_t ei = cudaGraphInstantiate(&exec, g, 0);
      cudaGraphDestroy(g);
      if (ei != cudaSuccess) { exec = nullptr; msg = std::string("chunk graph: ") + cudaGetErrorString(ei); return DTC_ERR_CUDA; }
      launches = n;
    }
    DTC_CUDA(cudaGraphLaunch(exec, s));
    counter += launches;
    return DTC_OK;
  }
};

__device__ __forceinline__ int list_dom(const Tile& t) { return t.dom; }
__device__ __forceinline__ int list_dom(int64_t e) { return (int)(e >> kListShift); }
__device__ __forceinline__ int list_dom(int d) { return d; }

// dst = the entries of src whose domain is still active; *count += their number.  The order
// is kept inside a block of 256 entries (one atomic per block), not across blocks.
template <typename E>
__global__ void __launch_bounds__(256) k_compact(const E* __restrict__ src, int64_t n, const int* __restrict__ dom_active,
                                                 E* __restrict__ dst, int* __restrict__ count) {
  __shared__ int wbase[8];
  __shared__ int base;
  const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  E e{};
  bool keep = false;
  if (i < n) {
    e = src[i];
    keep = dom_active[list_dom(e)] != 0;
  }
  const unsigned ballot = __ballot_sync(0xffffffffu, keep);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) wbase[warp] = __popc(ballot);
  __syncthreads();
  if (threadIdx.x == 0) {
    int tot = 0;
    for (int k = 0; k < 8; ++k) {
      const int c = wbase[k];
      wbase[k] = tot;
      tot += c;
    }
    base = tot ? atomicAdd(count, tot) : 0;
  }
  __syncthreads();
  if (keep) dst[base + wbase[warp] + __popc(ballot & ((1u << lane) - 1u))] = e;
}

template <typename E>
void launch_compact(const E* src, int64_t n, const int* act, E* dst, int* count, cudaStream_t s) {
  if (n > 0) k_compact<E><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, n, act, dst, count);
}

// The CG work lists restricted to the domains still iterating, so that the CTAs of converged
// domains are no longer launched (each launch of the full lists costs ~0.3 ms of immediately
// returning CTAs on a 512-domain batch).  From the original lists (W, and the multigrid lists
// of M when given) into the compacted copies (Wc; Pc counts and Mc pointers).
int compact_lists(DeviceSolver::Impl& I, const Work& W, const MgDev* M, const int* act, Work& Wc, MgPlan* Pc,
                  MgDev* Mc, int64_t& launches, std::string& msg) {
  cudaStream_t s = I.stream;
  static const MgPlan kNoLevels;
  const MgPlan& P = M ? *M->P : kNoLevels;
  const int nseg = 4 + 5 * P.nlev;
  int e;
  if ((e = ensure(I, bCompactCnt, sizeof(int) * nseg, msg))) return e;
  if ((e = ensure(I, bTilesIc, sizeof(Tile) * std::max<int64_t>(W.nti, 1), msg))) return e;
  if ((e = ensure(I, bTilesWc, sizeof(Tile) * std::max<int64_t>(W.ntw, 1), msg))) return e;
  if ((e = ensure(I, bNodesIc, sizeof(int64_t) * std::max<int64_t>(W.nnodes, 1), msg))) return e;
  if ((e = ensure(I, bBricksIc, sizeof(Tile) * std::max<int64_t>(W.nbi, 1), msg))) return e;
  if ((e = ensure(I, bMgTilesC, sizeof(Tile) * std::max<size_t>(P.tiles.size(), 1), msg))) return e;
  if ((e = ensure(I, bMgListC, sizeof(int) * std::max<size_t>(P.lists.size(), 1), msg))) return e;
  if ((e = ensure(I, bMgNodesC, sizeof(int64_t) * std::max<size_t>(P.nodes_l.size(), 1), msg))) return e;
  int* cnt = B<int>(I, bCompactCnt);
  DTC_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * nseg, s));
  Tile* tc = B<Tile>(I, bTilesIc);
  Tile* wc = B<Tile>(I, bTilesWc);
  int64_t* nc = B<int64_t>(I, bNodesIc);
  Tile* bc = B<Tile>(I, bBricksIc);
  Tile* mt = B<Tile>(I, bMgTilesC);
  int* ml = B<int>(I, bMgListC);
  int64_t* mn = B<int64_t>(I, bMgNodesC);
  launch_compact(W.ti, W.nti, act, tc, cnt + 0, s);
  launch_compact(W.nodes, W.nnodes, act, nc, cnt + 1, s);
  launch_compact(W.bi, W.nbi, act, bc, cnt + 2, s);
  launch_compact(W.tw, W.ntw, act, wc, cnt + 3, s);
  for (int l = 0; l < P.nlev; ++l) {
    launch_compact(M->tiles + P.sm_off[l], P.sm_n[l], act, mt + P.sm_off[l], cnt + 4 + 5 * l, s);
    launch_compact(M->tiles + P.in_off[l], P.in_n[l], act, mt + P.in_off[l], cnt + 5 + 5 * l, s);
    launch_compact(M->lists + P.list_off[l], P.list_n[l], act, ml + P.list_off[l], cnt + 6 + 5 * l, s);
    launch_compact(M->nodes + P.nl_off[l], P.nl_n[l], act, mn + P.nl_off[l], cnt + 7 + 5 * l, s);
    launch_compact(M->tiles + P.sw_off[l], P.sw_n[l], act, mt + P.sw_off[l], cnt + 8 + 5 * l, s);
  }
  launches += nseg;
  if ((e = launch_check(msg))) return e;
  std::vector<int> h(nseg);
  DTC_CUDA(cudaMemcpyAsync(h.data(), cnt, sizeof(int) * nseg, cudaMemcpyDeviceToHost, s));
  DTC_CUDA(cudaStreamSynchronize(s));
  Wc.ti = tc; Wc.nti = h[0];
  Wc.nodes = nc; Wc.nnodes = h[1];
  Wc.bi = bc; Wc.nbi = h[2];
  Wc.tw = wc; Wc.ntw = h[3];
  if (M) {
    Mc->bricks0 = bc; Mc->nbricks0 = h[2];
    Mc->nodes0 = nc; Mc->nnodes0 = h[1];
    Mc->tiles = mt;
    Mc->lists = ml;
    Mc->nodes = mn;
    for (int l = 0; l < P.nlev; ++l) {
      Pc->sm_n[l] = h[4 + 5 * l];
      Pc->in_n[l] = h[5 + 5 * l];
      Pc->list_n[l] = h[6 + 5 * l];
      Pc->nl_n[l] = h[7 + 5 * l];
      Pc->sw_n[l] = h[8 + 5 * l];
    }
  }
  return DTC_OK;
}

template <typename T, bool BLOCK, int NEN>
int run_cg(DeviceSolver::Impl& I, int ndom, const Work& W, T* x, T* r, T* p, T* w, const T* dinv,
           double rtol, const double* floor_abs, int64_t max_it, int64_t& launches, std::string& msg) {
  cudaStream_t s = I.stream;
  // work lists: the full ones until half the domains have converged, then compacted copies
  Work Wc = W;
  int64_t listed = ndom;
  const DomDev* dd = B<DomDev>(I, bDoms);
  const uint8_t* fl = B<uint8_t>(I, bFlags);
  ColState* st = B<ColState>(I, bSt);
  double* pw = B<double>(I, bPw);
  double* zz = B<double>(I, bZz);
  double* zr = B<double>(I, bZr);
  int* act = B<int>(I, bDomAct);
  int* cnt = B<int>(I, bCount);
  DTC_CUDA(cudaMemsetAsync(zz, 0, sizeof(double) * ndom * kNLC, s));
  DTC_CUDA(cudaMemsetAsync(zr, 0, sizeof(double) * ndom * kNLC, s));
  DTC_CUDA(cudaMemsetAsync(pw, 0, sizeof(double) * ndom * kNLC, s));
  if (W.nti > 0)
    k_initial_dots<T, BLOCK><<<(unsigned)(3 * W.nti), kThreads, 0, s>>>(W.ti, dd, fl, dinv, r, zz, zr, nullptr);
  k_colstate_init<<<ndom, 32, 0, s>>>(st, zz, zr, act, rtol, floor_abs, nullptr);
  launches += 2;
  if (int e = launch_check(msg)) return e;
  const int chunk = 32;
  int h_count = 1;
  ChunkGraph graph;
  for (int64_t it = 0; it < max_it + 2 && h_count > 0; it += chunk) {
    const bool f32 = sizeof(T) == 4;
    const double vb = I.profile ? I.active_sum(I.dom_vec_bytes) * sizeof(T) : 0;
    const double mb = I.profile ? I.active_sum(I.dom_mv_bytes) * sizeof(T) : 0;
    const double mf = I.profile ? I.active_sum(I.dom_mv_flops) : 0;
    const Tile* ti = Wc.ti;
    const int64_t nti = Wc.nti;
    const dim3 grid((unsigned)(3 * std::max<int64_t>(nti, 1)));
    auto body = [&](int64_t& nl) {
      for (int k = 0; k < chunk; ++k) {
        if (nti > 0) {
          int q = I.begin(0);
          k_direction<T, BLOCK><<<grid, kThreads, 0, s>>>(ti, dd, fl, dinv, r, p, st, act);
          I.end(f32 ? kcDirection32 : kcDirection64, q, 3 * vb, 0);
          q = I.begin(0);
          if (sizeof(T) == 4 && NEN == 8 && I.tensor_matvec)
            launch_sweep_tc(kTcApply, ti, nti, dd, I.svox(), fl, nullptr, nullptr, (const float*)p,
                            (float*)w, 1.0f, 0.0f, pw, nullptr, act, B<int>(I, bErr), s);
          else
            apply_k<T, NEN, false, true>(Wc, dd, I.svox(), fl, p, w, 1.0, pw, act, s);
          I.end(f32 ? kcMatvec32 : kcMatvec64, q, mb, mf);
          q = I.begin(0);
          k_update<T, BLOCK><<<grid, kThreads, 0, s>>>(ti, dd, fl, dinv, x, r, p, w, st, pw, zz, zr, act);
          I.end(f32 ? kcUpdate32 : kcUpdate64, q, 6 * vb, 0);
          nl += 3;
        }
        const int q = I.begin(0);
        k_colstate<<<ndom, 32, 0, s>>>(st, pw, zz, zr, act, max_it, nullptr);
        I.end(kcColstate, q, 0, 0);
        nl += 1;
      }
    };
    if (int e = graph.run(s, I.profile || !I.graphs, launches, body, msg)) return e;
    k_count_active<<<1, 256, 0, s>>>(act, ndom, cnt);
    launches += 1;
    if (int e = launch_check(msg)) return e;
    DTC_CUDA(cudaMemcpyAsync(&h_count, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (I.profile) {
      I.h_active.resize(ndom);
      DTC_CUDA(cudaMemcpyAsync(I.h_active.data(), act, sizeof(int) * ndom, cudaMemcpyDeviceToHost, s));
    }
    DTC_CUDA(cudaStreamSynchronize(s));
    I.flush();
    if (h_count > 0 && 2 * (int64_t)h_count <= listed) {
      if (int e = compact_lists(I, W, nullptr, act, Wc, nullptr, nullptr, launches, msg)) return e;
      graph.reset();
      listed = h_count;
    }
  }
  I.h_active.clear();
  return DTC_OK;
}


// FP32 CG preconditioned by one multigrid V-cycle per iteration (same column state machine
// and stopping rule as run_cg, with z = B r in place of the Jacobi z).
template <int NEN>
int run_cg_mg(DeviceSolver::Impl& I, int ndom, const Work& W, const MgDev& M, float* x, float* r, float* p, float* w,
              double rtol, const double* floor_abs, int64_t max_it, int64_t& launches, std::string& msg) {
  cudaStream_t s = I.stream;
  // work lists: the full ones until half the domains have converged, then compacted copies
  Work Wc = W;
  MgPlan Pc;   // offsets and counts of the multigrid lists (no bulk data)
  Pc.nlev = M.P->nlev; Pc.omega = M.P->omega; Pc.omega0 = M.P->omega0;
  Pc.sm_off = M.P->sm_off; Pc.sm_n = M.P->sm_n; Pc.in_off = M.P->in_off; Pc.in_n = M.P->in_n;
  Pc.sw_off = M.P->sw_off; Pc.sw_n = M.P->sw_n;
  Pc.list_off = M.P->list_off; Pc.list_n = M.P->list_n;
  Pc.nl_off = M.P->nl_off; Pc.nl_n = M.P->nl_n;
  MgDev Mc = M;
  Mc.P = &Pc;
  int64_t listed = ndom;   // domains the current lists were compacted to
  const DomDev* dd = B<DomDev>(I, bDoms);
  const uint8_t* fl = B<uint8_t>(I, bFlags);
  ColState* st = B<ColState>(I, bSt);
  double* pw = B<double>(I, bPw);
  double* zz = B<double>(I, bZz);
  double* zr = B<double>(I, bZr);
  int* act = B<int>(I, bDomAct);
  int* cnt = B<int>(I, bCount);
  float* dirf = B<float>(I, bDirF);      // per column: direction factor (NaN: column stopped)
  float* alphaf = B<float>(I, bAlphaF);  // per column: step length of the current iteration
  DTC_CUDA(cudaMemsetAsync(zz, 0, sizeof(double) * ndom * kNLC, s));
  DTC_CUDA(cudaMemsetAsync(zr, 0, sizeof(double) * ndom * kNLC, s));
  DTC_CUDA(cudaMemsetAsync(pw, 0, sizeof(double) * ndom * kNLC, s));
  mg_vcycle(I, M, 0, r, zz, zr, nullptr, launches);
  k_colstate_init<<<ndom, 32, 0, s>>>(st, zz, zr, act, rtol, floor_abs, dirf);
  k_count_active<<<1, 256, 0, s>>>(act, ndom, cnt);
  launches += 2;
  if (int e = launch_check(msg)) return e;
  const int chunk = 16;
  int h_count = 1;
  DTC_CUDA(cudaMemcpyAsync(&h_count, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
  DTC_CUDA(cudaStreamSynchronize(s));
  // a later refinement pass often starts with few domains still refining: lists to those
  if (h_count > 0 && 2 * (int64_t)h_count <= listed) {
    if (int e = compact_lists(I, W, &M, act, Wc, &Pc, &Mc, launches, msg)) return e;
    listed = h_count;
  }
  ChunkGraph graph;
  for (int64_t it = 0; it < max_it + 2 && h_count > 0; it += chunk) {
    const double vb = I.profile ? I.active_sum(I.dom_vec_bytes) * sizeof(float) : 0;
    const double mb = I.profile ? I.active_sum(I.dom_mv_bytes) * sizeof(float) : 0;
    const double mf = I.profile ? I.active_sum(I.dom_mv_flops) : 0;
    const int64_t nitems = 6 * Wc.nnodes;
    const unsigned gflat = (unsigned)std::max<int64_t>((nitems + 255) / 256, 1);
    auto body = [&](int64_t& nl) {
      for (int k = 0; k < chunk; ++k) {
        if (Wc.nti > 0) {
          int q = I.begin(0);
          k_direction_flat<<<gflat, 256, 0, s>>>(Wc.nodes, nitems, Mc.z0, p, dirf, act);
          I.end(kcDirection32, q, 3 * vb, 0);
          q = I.begin(0);
          if (NEN == 8 && I.tensor_matvec)
            launch_sweep_tc(kTcApply, Wc.ti, Wc.nti, dd, I.svox(), fl, nullptr, nullptr, p, w, 1.0f, 0.0f,
                            pw, nullptr, act, B<int>(I, bErr), s);
          else
            apply_k<float, NEN, false, true>(Wc, dd, I.svox(), fl, p, w, 1.0, pw, act, s);
          I.end(kcMatvec32, q, mb, mf);
          q = I.begin(0);
          k_alpha<<<ndom, 32, 0, s>>>(st, pw, alphaf, act);
          k_update_flat<<<gflat, 256, 0, s>>>(Wc.nodes, nitems, x, r, p, w, alphaf, Mc.binv0, Pc.omega0, Mc.t0, act);
          I.end(kcUpdate32, q, 7 * vb + vb / 12, 0);
          mg_vcycle(I, Mc, 0, r, zz, zr, act, nl, true);
          nl += 4;
        }
        const int q = I.begin(0);
        k_colstate<<<ndom, 32, 0, s>>>(st, pw, zz, zr, act, max_it, dirf);
        I.end(kcColstate, q, 0, 0);
        nl += 1;
      }
    };
    if (int e = graph.run(s, I.profile || !I.graphs, launches, body, msg)) return e;
    k_count_active<<<1, 256, 0, s>>>(act, ndom, cnt);
    launches += 1;
    if (int e = launch_check(msg)) return e;
    DTC_CUDA(cudaMemcpyAsync(&h_count, cnt, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (I.profile) {
      I.h_active.resize(ndom);
      DTC_CUDA(cudaMemcpyAsync(I.h_active.data(), act, sizeof(int) * ndom, cudaMemcpyDeviceToHost, s));
    }
    DTC_CUDA(cudaStreamSynchronize(s));
    I.flush();
    if (h_count > 0 && 2 * (int64_t)h_count <= listed) {
      if (int e = compact_lists(I, W, &M, act, Wc, &Pc, &Mc, launches, msg)) return e;
      graph.reset();
      listed = h_count;
    }
  }
  I.h_active.clear();
  return DTC_OK;
}
}  // namespace

// Host side of one device pass: the packed voxel factors, domain records and work lists of
// the solvable tasks, and the multigrid plan of a mixed multigrid solve.  Built by
// DeviceSolver::prepare, which touches no device state (it may run on a host thread while the
// solver executes an earlier pass), and consumed by DeviceSolver::solve.
// -------------------------------------------------------------------------------------
// Autotuner of the fine-level HEX08 sweeps (mixed_matvec = 2): the SIMT slab sweep and the
// tcgen05 sweep run the post-smoothing step of the batch's first V-cycle on its own tiles,
// one warm-up and three timed launches each (CUDA events on the solver stream); the faster
// one serves the whole solve (CG operator, residual and post-smoothing sweeps share the
// contraction).  Choices are cached per device and size class -- the median domain edge
// (16, 24, 32, 48, 64 voxels ...) and the kept-voxel fraction (below 0.15, 0.30, above) --
// so later batches of the same class skip the timing.
struct TuneKey {
  int device, nen, lclass, fclass;
  bool operator<(const TuneKey& o) const {
    return std::tie(device, nen, lclass, fclass) < std::tie(o.device, o.nen, o.lclass, o.fclass);
  }
};
struct TuneResult {
  int pick;            // 0 = SIMT, 1 = tensor cores
  float ms[2];         // the timed launches of each candidate (post-smoothing; SIMT at 6 CTAs/SM)
  // HEX08 SIMT slab sweeps: CTAs per SM of the residual, post-smoothing and CG application
  // sweeps, and the timed launches at 6 and 8 CTAs per SM (index 0 / 1)
  int minb[3] = {6, 6, 6};
  float shape_ms[3][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneResult> g_tune_choice;
constexpr int kTuneReps = 3;

// the decision in the solve's kernel statistics (also on a cache hit: the timings that decided)
void record_tuning(SolverStats& st, const TuneResult& r) {
  st.kc[kcTuneSimt].launches += kTuneReps;
  st.kc[kcTuneSimt].ms += r.ms[0];
  st.kc[kcTuneTc].launches += kTuneReps;
  st.kc[kcTuneTc].ms += r.ms[1];
  const int cls[3][2] = {{kcTuneRes4, kcTuneRes5}, {kcTuneSimt, kcTunePost5}, {kcTuneApply4, kcTuneApply5}};
  for (int k = 0; k < 3; ++k)
    for (int v = 0; v < 2; ++v)
      if (r.shape_ms[k][v] > 0.f && !(k == 1 && v == 0)) {
        st.kc[cls[k][v]].launches += kTuneReps;
        st.kc[cls[k][v]].ms += r.shape_ms[k][v];
      }
}

// CUDA-event time of kTuneReps launches after one untimed launch.
template <class F>
int time_launches(cudaStream_t s, F&& launch, float& ms, std::string& msg) {
  cudaEvent_t ev[2];
  DTC_CUDA(cudaEventCreate(&ev[0]));
  DTC_CUDA(cudaEventCreate(&ev[1]));
  launch();
  cudaEventRecord(ev[0], s);
  for (int r = 0; r < kTuneReps; ++r) launch();
  cudaEventRecord(ev[1], s);
  const cudaError_t ec = cudaEventSynchronize(ev[1]);
  if (ec == cudaSuccess) cudaEventElapsedTime(&ms, ev[0], ev[1]);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (ec != cudaSuccess) {
    msg = std::string("autotune: ") + cudaGetErrorString(ec);
    return DTC_ERR_CUDA;
  }
  return launch_check(msg);
}

TuneKey tune_key(int device, int nen, const std::vector<DomDev>& doms, const std::vector<float>& svox) {
  std::vector<int> Ls;
  for (const DomDev& D : doms) Ls.push_back(std::max(D.L[0], std::max(D.L[1], D.L[2])));
  std::nth_element(Ls.begin(), Ls.begin() + Ls.size() / 2, Ls.end());
  const int lmed = Ls.empty() ? 0 : Ls[Ls.size() / 2];
  int64_t kept = 0;
  for (float v : svox) kept += v != 0.0f;
  const double frac = svox.empty() ? 0.0 : (double)kept / (double)svox.size();
  return TuneKey{device, nen, (int)std::lround(4.0 * std::log2(std::max(lmed, 1))), frac < 0.15 ? 0 : frac < 0.30 ? 1 : 2};
}

// The fine-level operator of an FP32 multigrid solve, chosen per device, element type and size
// class (median domain edge in quarter octaves, kept-voxel fraction below 0.15 / 0.30 / above)
// by CUDA-event timings on the batch's own tiles and vectors:
//  * HEX08: the SIMT slab sweep or the tcgen05 sweep (timed on the post-smoothing sweep); for
//    the SIMT sweep also the register budget of each of its three kernels -- residual,
//    post-smoothing, CG application -- at 6 CTAs per SM (80 registers) or 8 (64);
//  * HEX20: the SIMT brick kernel or the tcgen05 brick kernel (the operator of the residual and
//    post-smoothing steps and of the CG application).
int autotune_sweep(DeviceSolver::Impl& I, SolverStats& st, Work& W, MgDev& M, const std::vector<DomDev>& doms,
                   const std::vector<float>& svox, int nen, std::string& msg) {
  cudaStream_t s = I.stream;
  const TuneKey key = tune_key(I.device, nen, doms, svox);
  auto adopt = [&](const TuneResult& r) {
    I.tensor_matvec = r.pick == 1;
    M.minb_res = r.minb[0];
    M.minb_post = r.minb[1];
    W.minb32 = r.minb[2];
    record_tuning(st, r);
  };
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_choice.find(key);
    if (it != g_tune_choice.end()) {
      adopt(it->second);
      return DTC_OK;
    }
  }
  const int64_t nsm = M.P->sm_n[0];
  const Tile* tsm = M.tiles + M.P->sm_off[0];
  if (nsm <= 0 || (nen == 20 && (M.nbricks0 <= 0 || !W.ke20tc))) return DTC_OK;
  const float* b = B<float>(I, bR32);
  double* zz = B<double>(I, bZz);
  double* zr = B<double>(I, bZr);
  const unsigned g = (unsigned)(3 * nsm);
  const Tile* tsw = M.tiles + M.P->sw_off[0];
  const unsigned gw = (unsigned)(3 * M.P->sw_n[0]);
  TuneResult r{0, {0.f, 0.f}};
  int e;
  for (int cand = 0; cand < 2; ++cand) {
    auto launch = [&]() {
      if (nen == 20) {
        if (cand == 0)
          launch_ebe<float, 20, false, false>(M.bricks0, M.nbricks0, M.doms0, M.svox0, M.flags0, M.ke32, M.t0, M.z0,
                                              -1.0, nullptr, nullptr, s);
        else
          launch_ebe_tc(M.bricks0, M.nbricks0, M.doms0, M.svox0, M.flags0, W.ke20tc, M.t0, M.z0, -1.0, nullptr,
                        nullptr, M.err, s);
      } else if (cand == 0) {
        launch_mg_matvec<kMgPost, true>(4, gw, s, tsw, M.doms0, M.svox0, M.binv0, b, M.t0, M.z0, M.P->omega0, zz,
                                        zr, nullptr);
      } else {
        launch_sweep_tc(kTcPost, tsm, nsm, M.doms0, M.svox0, M.flags0, M.binv0, b, M.t0, M.z0, 1.0f, M.P->omega0, zz,
                        zr, nullptr, M.err, s);
      }
    };
    if ((e = time_launches(s, launch, r.ms[cand], msg))) return e;
  }
  r.pick = r.ms[1] < r.ms[0] ? 1 : 0;
  if (nen == 8 && r.pick == 0) {
    // register budgets of the three SIMT sweeps (the post-smoothing at 6 CTAs/SM is ms[0])
    r.shape_ms[1][0] = r.ms[0];
    for (int v = 0; v < 2; ++v) {
      const int minb = v == 0 ? 6 : 8;
      auto res = [&]() {
        launch_mg_matvec<kMgRes, false>(minb, gw, s, tsw, M.doms0, M.svox0, M.binv0, b, M.t0, M.z0, M.P->omega0,
                                        nullptr, nullptr, nullptr);
      };
      if ((e = time_launches(s, res, r.shape_ms[0][v], msg))) return e;
      if (v == 1) {
        auto post = [&]() {
          launch_mg_matvec<kMgPost, true>(minb, gw, s, tsw, M.doms0, M.svox0, M.binv0, b, M.t0, M.z0, M.P->omega0,
                                          zz, zr, nullptr);
        };
        if ((e = time_launches(s, post, r.shape_ms[1][v], msg))) return e;
      }
      Work Wv = W;
      Wv.minb32 = minb;
      auto apply = [&]() {
        apply_k<float, 8, false, true>(Wv, M.doms0, M.svox0, M.flags0, M.t0, M.z0, 1.0, zz, nullptr, s);
      };
      if ((e = time_launches(s, apply, r.shape_ms[2][v], msg))) return e;
    }
    for (int k = 0; k < 3; ++k) r.minb[k] = r.shape_ms[k][1] < r.shape_ms[k][0] ? 8 : 6;
  }
  adopt(r);
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune_choice[key] = r;
  return DTC_OK;
}

// The register budget of the HEX08 FP64 slab sweep (outer residual, reactions, plain FP64 CG):
// 4 CTAs per SM (128 registers) or 6 (80), timed on the batch's interior tiles (X -> R64, which
// the solve overwrites next), cached per class like the FP32 choice.
struct Tune64 { int minb; float ms[2]; };
std::map<TuneKey, Tune64> g_tune64;

int autotune_fp64(DeviceSolver::Impl& I, SolverStats& st, Work& W, const std::vector<DomDev>& doms,
                  const std::vector<float>& svox, const double* X, double* R64, std::string& msg) {
  const TuneKey key = tune_key(I.device, 8, doms, svox);
  Tune64 r{4, {0.f, 0.f}};
  bool cached = false;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune64.find(key);
    if (it != g_tune64.end()) { r = it->second; cached = true; }
  }
  if (!cached && W.nti > 0) {
    for (int v = 0; v < 2; ++v) {
      Work Wv = W;
      Wv.minb64 = v == 0 ? 4 : 6;
      auto launch = [&]() {
        apply_k<double, 8, false, false>(Wv, B<DomDev>(I, bDoms), I.svox(), B<uint8_t>(I, bFlags), X, R64,
                                         -1.0, nullptr, nullptr, I.stream);
      };
      if (int e = time_launches(I.stream, launch, r.ms[v], msg)) return e;
    }
    r.minb = r.ms[1] < r.ms[0] ? 6 : 4;
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune64[key] = r;
  }
  W.minb64 = r.minb;
  for (int v = 0; v < 2; ++v) {
    st.kc[v == 0 ? kcTuneF64a : kcTuneF64b].launches += kTuneReps;
    st.kc[v == 0 ? kcTuneF64a : kcTuneF64b].ms += r.ms[v];
  }
  return DTC_OK;
}

struct HostBatch {
  int nen = 0;
  std::vector<int64_t> tidx;   // tasks solved in this pass
  std::vector<DomDev> doms;
  std::vector<Tile> tiles_i, tiles_a, bricks_i, bricks_a;
  std::vector<Tile> tiles_w;   // interior sweep tiles (rows of kSweepX nodes)
  std::vector<int64_t> nodes_i;
  std::vector<float> svox;
  int64_t node_total = 0;
  std::vector<double> dom_vec, dom_mv, dom_fl;   // per-domain algorithmic work of one launch
  bool has_mg = false;
  MgPlan mg;
  double ms_pack = 0, ms_mg = 0;
  int up_slot = -1;   // device slot its voxel factors were uploaded to (DeviceSolver::upload_voxels)
};
void HostBatchDeleter::operator()(HostBatch* p) const { delete p; }

template <int NEN>
int prepare_nen(std::vector<DomainTask>& tasks, const dtc_options& opt, double nu, HostBatch& hb) {
  const auto tpack = std::chrono::steady_clock::now();
  using EL = Elem<NEN>;
  constexpr int m = EL::M;
  std::vector<DomDev>& doms = hb.doms;
  std::vector<Tile>&tiles_i = hb.tiles_i, &tiles_a = hb.tiles_a, &bricks_i = hb.bricks_i, &bricks_a = hb.bricks_a;
  std::vector<int64_t>& nodes_i = hb.nodes_i;
  std::vector<float>& svox = hb.svox;
  std::vector<int64_t>& tidx = hb.tidx;
  int64_t& node_total = hb.node_total;
  // which tasks are solved here, and each domain's voxel and node offsets (serial, cheap)
  for (size_t k = 0; k < tasks.size(); ++k)
    if (tasks[k].plan->status == DTC_DOMAIN_OK) tidx.push_back((int64_t)k);
  const int ndom_p = (int)tidx.size();
  std::vector<int64_t> vox_offs(ndom_p), node_offs(ndom_p);
  int64_t vox_total = 0;
  for (int d = 0; d < ndom_p; ++d) {
    const dtc_domain_in& in = *tasks[tidx[d]].in;
    vox_offs[d] = vox_total;
    node_offs[d] = node_total;
    vox_total += in.L[0] * in.L[1] * in.L[2];
    node_total += (int64_t)(m * in.L[0] + 1) * (m * in.L[1] + 1) * (m * in.L[2] + 1);
  }
  svox.assign((size_t)vox_total, 0.f);
  // per domain: voxel factors, node activity and work lists (host threads)
  struct Packed {
    DomDev D;
    std::vector<Tile> ti, ta, bi, ba, tw;
    std::vector<int64_t> ni;
    double vec = 0, mv = 0, fl = 0;
  };
  std::vector<Packed> packed(ndom_p);
  auto pack_one = [&](int dom, Packed& out) {
    const size_t k = (size_t)tidx[dom];
    DomainTask& t = tasks[k];
    const MeshPlan& mp = *t.plan;
    const dtc_domain_in& in = *t.in;
    DomDev D{};
    D.m = m;
    for (int d = 0; d < 3; ++d) { D.L[d] = (int32_t)in.L[d]; D.n[d] = m * (int32_t)in.L[d] + 1; }
    D.vox_off = vox_offs[dom];
    D.node_off = node_offs[dom];
    D.delta = in.delta[0];
    for (int d = 0; d < 3; ++d) {
      D.min_c_off[d] = in.xa_n[d] - 1;
      D.min_c[d] = (double)(in.xa_n[d] - 1) * in.delta[d];
      D.max_c[d] = (double)(in.xa_n[d] + in.L[d] - 1) * in.delta[d];
    }
    const int64_t nvox = in.L[0] * in.L[1] * in.L[2];
    const double a = in.phdsize[0] * in.delta[0];
    D.scale = in.E_voxel ? a : a * in.E;
    float* sv = svox.data() + D.vox_off;
    for (int64_t v = 0; v < nvox; ++v) sv[v] = mp.kept[v] ? (in.E_voxel ? in.E_voxel[v] : 1.0f) : 0.0f;
    // node activity on the (fine) grid for the work lists; kept voxels per node for the flop count
    const int nx = D.n[0], ny = D.n[1], nz = D.n[2];
    std::vector<uint8_t> act((size_t)nx * ny * nz, 0);
    double kept = 0;
    int64_t v = 0;
    for (int vz = 0; vz < (int)in.L[2]; ++vz)
      for (int vy = 0; vy < (int)in.L[1]; ++vy)
        for (int vx = 0; vx < (int)in.L[0]; ++vx, ++v) {
          if (sv[v] == 0.0f) continue;
          kept += 1;
          for (int c = 0; c <= m; ++c)
            for (int b2 = 0; b2 <= m; ++b2)
              for (int a2 = 0; a2 <= m; ++a2) {
                const int odd = (a2 == 1) + (b2 == 1) + (c == 1);
                if (m == 2 && odd > 1) continue;   // HEX20 has no face or body nodes
                act[(m * vx + a2) + (size_t)nx * ((m * vy + b2) + (size_t)ny * (m * vz + c))] = 1;
              }
        }
    // algorithmic work of one launch on this domain, in elements of T per vector (bytes later)
    // and flops: vector kernels touch 72 values per active interior node per vector; the
    // stiffness application reads the input and writes the output (2 vectors) plus one
    // float per voxel, and costs 2 * (3 NEN)^2 flops per kept voxel and load case.
    // the active interior nodes (flat vector kernels of the multigrid path) in one pass
    out.ni.reserve((size_t)kept * (m == 1 ? 2 : 8) + 64);
    for (int z = 1; z < nz - 1; ++z)
      for (int y = 1; y < ny - 1; ++y) {
        const size_t row = (size_t)nx * (y + (size_t)ny * z);
        for (int x = 1; x < nx - 1; ++x)
          if (act[x + row])
            out.ni.push_back(((int64_t)dom << kListShift) | (D.node_off + x + (int64_t)row));
      }
    {
      const double nint = (double)out.ni.size();
      out.vec = 72.0 * nint;
      out.mv = 2 * 72.0 * nint + (double)nvox;
      out.fl = kept * 2.0 * (3 * NEN) * (3 * NEN) * kNLC;
    }
    auto any_active = [&](int x0, int y0, int z0, int sx, int sy, int sz, int lo, int hx, int hy, int hz) {
      for (int z = std::max(z0, lo); z < std::min(z0 + sz, hz + 1); ++z)
        for (int y = std::max(y0, lo); y < std::min(y0 + sy, hy + 1); ++y)
          for (int x = std::max(x0, lo); x < std::min(x0 + sx, hx + 1); ++x)
            if (act[x + (size_t)nx * (y + (size_t)ny * z)]) return true;
      return false;
    };
    // node tiles (vector kernels) over the interior / all nodes
    for (int z0 = 1; z0 <= nz - 2; z0 += kTileZ)
      for (int y0 = 1; y0 <= ny - 2; y0 += kTileY)
        for (int x0 = 1; x0 <= nx - 2; x0 += kTileX)
          if (any_active(x0, y0, z0, kTileX, kTileY, kTileZ, 1, nx - 2, ny - 2, nz - 2))
            out.ti.push_back(Tile{dom, (int16_t)x0, (int16_t)y0, (int16_t)z0, 0});
    // sweep tiles (the slab sweeps over the interior): rows of kSweepX nodes
    for (int z0 = 1; z0 <= nz - 2; z0 += kTileZ)
      for (int y0 = 1; y0 <= ny - 2; y0 += kTileY)
        for (int x0 = 1; x0 <= nx - 2; x0 += kSweepX)
          if (any_active(x0, y0, z0, kSweepX, kTileY, kTileZ, 1, nx - 2, ny - 2, nz - 2))
            out.tw.push_back(Tile{dom, (int16_t)x0, (int16_t)y0, (int16_t)z0, 0});
    for (int z0 = 0; z0 <= nz - 1; z0 += kTileZ)
      for (int y0 = 0; y0 <= ny - 1; y0 += kTileY)
        for (int x0 = 0; x0 <= nx - 1; x0 += kTileX)
          if (any_active(x0, y0, z0, kTileX, kTileY, kTileZ, 0, nx - 1, ny - 1, nz - 1))
            out.ta.push_back(Tile{dom, (int16_t)x0, (int16_t)y0, (int16_t)z0, 0});
    // voxel bricks (HEX20 operator): brick origin in voxels, owned nodes m*origin + [0, m*B)
    for (int bz = 0; NEN == 20 && m * bz <= nz - 1; bz += EL::BZ)
      for (int by = 0; m * by <= ny - 1; by += EL::BY)
        for (int bx = 0; m * bx <= nx - 1; bx += EL::BX) {
          const int ox = m * bx, oy = m * by, oz = m * bz;
          if (any_active(ox, oy, oz, m * EL::BX, m * EL::BY, m * EL::BZ, 1, nx - 2, ny - 2, nz - 2))
            out.bi.push_back(Tile{dom, (int16_t)bx, (int16_t)by, (int16_t)bz, 0});
          if (any_active(ox, oy, oz, m * EL::BX, m * EL::BY, m * EL::BZ, 0, nx - 1, ny - 1, nz - 1))
            out.ba.push_back(Tile{dom, (int16_t)bx, (int16_t)by, (int16_t)bz, 0});
        }
    out.D = D;
  };
  parallel_for(ndom_p, opt.host_threads, [&](int64_t d) { pack_one((int)d, packed[d]); });
  // concatenate in domain order
  for (int d = 0; d < ndom_p; ++d) {
    Packed& q = packed[d];
    doms.push_back(q.D);
    tiles_i.insert(tiles_i.end(), q.ti.begin(), q.ti.end());
    tiles_a.insert(tiles_a.end(), q.ta.begin(), q.ta.end());
    hb.tiles_w.insert(hb.tiles_w.end(), q.tw.begin(), q.tw.end());
    bricks_i.insert(bricks_i.end(), q.bi.begin(), q.bi.end());
    bricks_a.insert(bricks_a.end(), q.ba.begin(), q.ba.end());
    nodes_i.insert(nodes_i.end(), q.ni.begin(), q.ni.end());
    hb.dom_vec.push_back(q.vec);
    hb.dom_mv.push_back(q.mv);
    hb.dom_fl.push_back(q.fl);
  }
  hb.ms_pack = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tpack).count();
  // multigrid plan of the mixed inner solve (HEX08 levels; HEX20 starts with p-coarsening)
  if (opt.precision == DTC_PREC_MIXED && opt.inner_precond == 2 && !tiles_i.empty()) {
    const auto tb = std::chrono::steady_clock::now();
    build_mg(hb.mg, doms, svox, tiles_i, hb.tiles_w, nu, NEN, opt.host_threads);
    hb.has_mg = true;
    hb.ms_mg = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count();
  }
  return DTC_OK;
}

template <int NEN>
int solve_nen(DeviceSolver::Impl& I, SolverStats& stats_, std::vector<DomainTask>& tasks, const dtc_options& opt,
              double nu, int keep, HostBatch& hb, std::string& msg) {
  DTC_CUDA(cudaSetDevice(I.device));
  cudaStream_t s = I.stream;
  stats_ = SolverStats();
  static const char* kNames[kcNumClasses] = {"matvec_f32", "matvec_f64", "update_f32", "update_f64",
                                             "direction_f32", "direction_f64", "colstate", "reaction_f64",
                                             "project_f64", "mg_jacobi_f32", "mg_residual_f32",
                                             "mg_postsmooth_f32", "mg_transfer_f32", "mg_coarse_levels_f32",
                                             "rotation_search_f64", "autotune_simt_sweep", "autotune_tc_sweep",
                                             "autotune_res_sweep_6cta", "autotune_res_sweep_8cta",
                                             "autotune_post_sweep_8cta", "autotune_apply_sweep_6cta",
                                             "autotune_apply_sweep_8cta", "autotune_f64_sweep_4cta",
                                             "autotune_f64_sweep_6cta", "host_pack", "host_multigrid_build"};
  for (int c = 0; c < kcNumClasses; ++c) stats_.kc[c].name = kNames[c];
  I.stats = &stats_;
  I.profile = opt.profile_kernels != 0;
  I.tensor_matvec = opt.mixed_matvec == 1;
  const bool tune = opt.mixed_matvec == 2;
  I.graphs = opt.graph_chunks == 0;
  I.pending.clear();
  I.h_active.clear();
  I.dom_mv_bytes.clear(); I.dom_mv_flops.clear(); I.dom_vec_bytes.clear();
  // constant tables
  {
    double kh[576];
    float kh32[576];
    voxel_stiffness(8, nu, kh);
    for (int i = 0; i < 576; ++i) kh32[i] = (float)kh[i];
    DTC_CUDA(cudaMemcpyToSymbolAsync(c_khat64, kh, sizeof(kh), 0, cudaMemcpyHostToDevice, s));
    DTC_CUDA(cudaMemcpyToSymbolAsync(c_khat32, kh32, sizeof(kh32), 0, cudaMemcpyHostToDevice, s));
    float2 khr[4 * 3 * 24];
    for (int b = 0; b < 2; ++b)
      for (int c = 0; c < 2; ++c) {
        const int l0 = corner_local(0, 1 - b, 1 - c), l1 = corner_local(1, 1 - b, 1 - c);
        for (int r = 0; r < 3; ++r)
          for (int col = 0; col < 24; ++col)
            khr[((2 * b + c) * 3 + r) * 24 + col] = make_float2(kh32[col * 24 + 3 * l0 + r], kh32[col * 24 + 3 * l1 + r]);
      }
    DTC_CUDA(cudaMemcpyToSymbolAsync(c_khat32r2, khr, sizeof(khr), 0, cudaMemcpyHostToDevice, s));
    if (int e = upload_tc_operand(kh, s, msg)) return e;
    if (I.tensor_matvec || tune) {
      if (int e = set_tc_spin_limit(opt.tc_wait_spins, s, msg)) return e;
      if (int e = allow_sweep_tc(msg)) return e;
    }
    if (NEN == 20) {
      std::vector<double> k20(3600);
      std::vector<float> k20f(3600);
      voxel_stiffness(20, nu, k20.data());
      for (int i = 0; i < 3600; ++i) k20f[i] = (float)k20[i];
      DTC_CUDA(cudaMemcpyToSymbolAsync(c_k20_64, k20.data(), sizeof(double) * 3600, 0, cudaMemcpyHostToDevice, s));
      // the element kernel stages the matrix from global memory: FP64 then FP32 copy
      if (int e = ensure(I, bKe20, sizeof(double) * 3600 + sizeof(float) * 3600, msg)) return e;
      DTC_CUDA(cudaMemcpyAsync(I.bufs[bKe20], k20.data(), sizeof(double) * 3600, cudaMemcpyHostToDevice, s));
      DTC_CUDA(cudaMemcpyAsync(B<double>(I, bKe20) + 3600, k20f.data(), sizeof(float) * 3600, cudaMemcpyHostToDevice,
                               s));
      if (I.tensor_matvec || tune) {   // HEX20 FP32 applications on the tensor cores
        std::vector<float> img(tc20_operand_bytes() / sizeof(float));
        build_tc20_operand(k20.data(), img.data());
        if (int e = ensure(I, bKe20tc, tc20_operand_bytes(), msg)) return e;
        DTC_CUDA(cudaMemcpyAsync(I.bufs[bKe20tc], img.data(), tc20_operand_bytes(), cudaMemcpyHostToDevice, s));
        if (int e = allow_ebe_tc(msg)) return e;
      }
      DTC_CUDA(cudaStreamSynchronize(s));   // the host vectors go out of scope
    }
    if constexpr (NEN == 20)
      if (int e = allow_all_ebe<NEN>(msg)) return e;   // per device, cheap
  }
  // the host side of the pass (prepare_nen)
  const auto tpack = std::chrono::steady_clock::now();
  std::vector<DomDev>& doms = hb.doms;
  std::vector<Tile>&tiles_i = hb.tiles_i, &tiles_a = hb.tiles_a, &bricks_i = hb.bricks_i, &bricks_a = hb.bricks_a;
  std::vector<int64_t>& nodes_i = hb.nodes_i;
  std::vector<float>& svox = hb.svox;
  const std::vector<int64_t>& tidx = hb.tidx;
  const int64_t node_total = hb.node_total;
  I.dom_vec_bytes = hb.dom_vec;
  I.dom_mv_bytes = hb.dom_mv;
  I.dom_mv_flops = hb.dom_fl;
  stats_.kc[kcHostPack].ms += hb.ms_pack;
  if (hb.has_mg) {
    stats_.kc[kcHostMgBuild].ms += hb.ms_mg;
    stats_.kc[kcHostMgBuild].launches += 1;
  }
  const int ndom = (int)doms.size();
  if (ndom == 0) return DTC_OK;
  const int64_t nti = (int64_t)tiles_i.size(), nta = (int64_t)tiles_a.size();
  const int64_t nbi = (int64_t)bricks_i.size(), nba = (int64_t)bricks_a.size();
  const size_t vbytes64 = sizeof(double) * node_total * 3 * kNLC, vbytes32 = sizeof(float) * node_total * 3 * kNLC;
  const bool mixed = opt.precision == DTC_PREC_MIXED;
  int e;
  if ((e = ensure(I, bDoms, sizeof(DomDev) * ndom, msg))) return e;
  if ((e = ensure(I, bTilesI, sizeof(Tile) * std::max<int64_t>(nti, 1), msg))) return e;
  if ((e = ensure(I, bTilesA, sizeof(Tile) * std::max<int64_t>(nta, 1), msg))) return e;
  const int64_t ntw = (int64_t)hb.tiles_w.size();
  if ((e = ensure(I, bTilesW, sizeof(Tile) * std::max<int64_t>(ntw, 1), msg))) return e;
  if ((e = ensure(I, bBricksI, sizeof(Tile) * std::max<int64_t>(nbi, 1), msg))) return e;
  if ((e = ensure(I, bBricksA, sizeof(Tile) * std::max<int64_t>(nba, 1), msg))) return e;
  I.svox_dev = nullptr;
  if (hb.up_slot < 0 && (e = ensure(I, bSvox, sizeof(float) * svox.size(), msg))) return e;
  if ((e = ensure(I, bFlags, node_total, msg))) return e;
  if ((e = ensure(I, bDinv64, sizeof(double) * node_total * 3, msg))) return e;
  if ((e = ensure(I, bDinv32, sizeof(float) * node_total * 3, msg))) return e;
  if ((e = ensure(I, bBinv32, sizeof(float) * node_total * 6, msg))) return e;
  if ((e = ensure(I, bX, vbytes64, msg))) return e;
  if ((e = ensure(I, bR64, vbytes64, msg))) return e;
  if (mixed) {
    if ((e = ensure(I, bR32, vbytes32, msg))) return e;
    if ((e = ensure(I, bX32, vbytes32, msg))) return e;
    if ((e = ensure(I, bP32, vbytes32, msg))) return e;
    if ((e = ensure(I, bW32, vbytes32, msg))) return e;
  } else {
    if ((e = ensure(I, bP64, vbytes64, msg))) return e;
    if ((e = ensure(I, bW64, vbytes64, msg))) return e;
  }
  const size_t ncol = (size_t)ndom * kNLC;
  if ((e = ensure(I, bSt, sizeof(ColState) * ncol, msg))) return e;
  if ((e = ensure(I, bOst, sizeof(ColState) * ncol, msg))) return e;
  if ((e = ensure(I, bPw, sizeof(double) * ncol, msg))) return e;
  if ((e = ensure(I, bZz, sizeof(double) * ncol, msg))) return e;
  if ((e = ensure(I, bZr, sizeof(double) * ncol, msg))) return e;
  if ((e = ensure(I, bTarget, sizeof(double) * ncol, msg))) return e;
  if ((e = ensure(I, bDirF, sizeof(float) * ncol, msg))) return e;
  if ((e = ensure(I, bAlphaF, sizeof(float) * ncol, msg))) return e;
  if ((e = ensure(I, bDomAct, sizeof(int) * ndom, msg))) return e;
  if ((e = ensure(I, bCount, sizeof(int), msg))) return e;
  // macro order 2 solves its 60 load cases as three column passes of 24 over the same batch
  const int order = opt.macro_order == 2 ? 2 : 1;
  const int nm = macro_nodes(order), nl = macro_loadcases(order);
  const int ncp = (nl + kNLC - 1) / kNLC;
  // the energy estimator's Gram matrix is ldg x ldg per domain (the passes' 24-column blocks);
  // the solutions of every pass but the last stay on the device for the cross-pass blocks
  const bool energy = opt.tensor_estimator == 1;
  const int ldg = kNLC * ncp;
  if ((e = ensure(I, bFf, sizeof(double) * std::max(nl * nl, energy ? ldg * ldg : 0) * ndom, msg))) return e;
  if (energy && ncp > 1 && (e = ensure(I, bXkeep, vbytes64 * (ncp - 1), msg))) return e;
  if ((e = ensure(I, bErr, sizeof(int), msg))) return e;
  DTC_CUDA(cudaMemsetAsync(I.bufs[bErr], 0, sizeof(int), s));

  stats_.kc[kcHostPack].ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tpack).count();
  stats_.kc[kcHostPack].launches += 1;
  auto t0 = std::chrono::steady_clock::now();
  DTC_CUDA(cudaMemcpyAsync(I.bufs[bDoms], doms.data(), sizeof(DomDev) * ndom, cudaMemcpyHostToDevice, s));
  if (nti) DTC_CUDA(cudaMemcpyAsync(I.bufs[bTilesI], tiles_i.data(), sizeof(Tile) * nti, cudaMemcpyHostToDevice, s));
  if (nta) DTC_CUDA(cudaMemcpyAsync(I.bufs[bTilesA], tiles_a.data(), sizeof(Tile) * nta, cudaMemcpyHostToDevice, s));
  if (ntw)
    DTC_CUDA(cudaMemcpyAsync(I.bufs[bTilesW], hb.tiles_w.data(), sizeof(Tile) * ntw, cudaMemcpyHostToDevice, s));
  if (nbi) DTC_CUDA(cudaMemcpyAsync(I.bufs[bBricksI], bricks_i.data(), sizeof(Tile) * nbi, cudaMemcpyHostToDevice, s));
  if ((e = ensure(I, bNodesI, sizeof(int64_t) * std::max<size_t>(nodes_i.size(), 1), msg))) return e;
  if (!nodes_i.empty())
    DTC_CUDA(cudaMemcpyAsync(I.bufs[bNodesI], nodes_i.data(), sizeof(int64_t) * nodes_i.size(), cudaMemcpyHostToDevice,
                             s));
  if (nba) DTC_CUDA(cudaMemcpyAsync(I.bufs[bBricksA], bricks_a.data(), sizeof(Tile) * nba, cudaMemcpyHostToDevice, s));
  if (hb.up_slot >= 0) {   // uploaded while the previous pass solved: order the solve after the copy
    DTC_CUDA(cudaStreamWaitEvent(s, I.up_ev[hb.up_slot], 0));
    I.svox_dev = I.up_dev[hb.up_slot];
  } else {
    DTC_CUDA(cudaMemcpyAsync(I.bufs[bSvox], svox.data(), sizeof(float) * svox.size(), cudaMemcpyHostToDevice, s));
  }
  DTC_CUDA(cudaMemsetAsync(I.bufs[bFlags], 0, node_total, s));
  DTC_CUDA(cudaMemsetAsync(I.bufs[bDinv64], 0, sizeof(double) * node_total * 3, s));
  DTC_CUDA(cudaMemsetAsync(I.bufs[bDinv32], 0, sizeof(float) * node_total * 3, s));
  DTC_CUDA(cudaMemsetAsync(I.bufs[bX], 0, vbytes64, s));
  DTC_CUDA(cudaMemsetAsync(I.bufs[bR64], 0, vbytes64, s));
  DTC_CUDA(cudaMemsetAsync(I.bufs[bFf], 0, sizeof(double) * std::max(nl * nl, energy ? ldg * ldg : 0) * ndom, s));
  // device time of the solve, inputs resident: from here (voxel factors and work lists
  // uploaded) to the last kernel, measured with CUDA events on the solver stream
  if (!I.ev_solve[0]) {
    DTC_CUDA(cudaEventCreate(&I.ev_solve[0]));
    DTC_CUDA(cudaEventCreate(&I.ev_solve[1]));
  }
  const Tile* ti = B<Tile>(I, bTilesI);
  const Tile* ta = B<Tile>(I, bTilesA);
  const double* ke64 = NEN == 20 ? B<double>(I, bKe20) : nullptr;
  const float* ke20tc = (NEN == 20 && (I.tensor_matvec || tune)) ? B<float>(I, bKe20tc) : nullptr;
  Work W{ti, ta, B<Tile>(I, bBricksI), B<Tile>(I, bBricksA), nti, nta, nbi, nba,
               B<int64_t>(I, bNodesI), (int64_t)nodes_i.size(), ke64,
               ke64 ? reinterpret_cast<const float*>(ke64 + 3600) : nullptr, ke20tc, B<int>(I, bErr)};
  W.tw = B<Tile>(I, bTilesW);
  W.ntw = ntw;
  const DomDev* dd = B<DomDev>(I, bDoms);
  uint8_t* fl = B<uint8_t>(I, bFlags);
  double* X = B<double>(I, bX);
  double* R64 = B<double>(I, bR64);
  int64_t& L = stats_.kernel_launches;
  // the FP64 sweep's register budget (its cost does not depend on the values: X is zero here,
  // R64 is scratch), before the solve's device time starts
  if (tune && NEN == 8 && (e = autotune_fp64(I, stats_, W, doms, svox, X, R64, msg))) return e;
  DTC_CUDA(cudaEventRecord(I.ev_solve[0], s));
  if (nta) {
    DTC_CUDA(cudaMemsetAsync(I.bufs[bBinv32], 0, sizeof(float) * node_total * 6, s));
    k_node_setup<NEN><<<(unsigned)nta, kThreads, 0, s>>>(ta, dd, I.svox(), fl, B<double>(I, bDinv64),
                                                    B<float>(I, bDinv32), B<float>(I, bBinv32));
    ++L;
  }
  if ((e = launch_check(msg))) return e;
  const dim3 gi((unsigned)(3 * std::max<int64_t>(nti, 1))), ga((unsigned)(3 * std::max<int64_t>(nta, 1)));
  ColState* ost = B<ColState>(I, bOst);
  const bool use_mg = mixed && opt.inner_precond == 2 && nti > 0;
  MgPlan mgp;
  MgDev mgd{};
  if (use_mg) {   // multigrid hierarchy: built on the host from the voxel factors, set up on the device
    if (hb.has_mg) {
      mgp = std::move(hb.mg);
    } else {
      const auto tb = std::chrono::steady_clock::now();
      build_mg(mgp, doms, svox, tiles_i, hb.tiles_w, nu, NEN, opt.host_threads);
      stats_.kc[kcHostMgBuild].ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tb).count();
      stats_.kc[kcHostMgBuild].launches += 1;
    }
    const int64_t cn = std::max<int64_t>(mgp.nodes, 1);
    if ((e = ensure(I, bZ32, vbytes32, msg)) || (e = ensure(I, bT32, vbytes32, msg)) ||
        (e = ensure(I, bMgDoms, sizeof(DomDev) * mgp.doms.size(), msg)) ||
        (e = ensure(I, bMgTiles, sizeof(Tile) * std::max<size_t>(mgp.tiles.size(), 1), msg)) ||
        (e = ensure(I, bMgSvox, sizeof(float) * std::max<size_t>(mgp.svox.size(), 1), msg)) ||
        (e = ensure(I, bMgFlags, cn, msg)) || (e = ensure(I, bMgDinv64, sizeof(double) * 3 * cn, msg)) ||
        (e = ensure(I, bMgDinv32, sizeof(float) * 3 * cn, msg)) ||
        (e = ensure(I, bMgBinv32, sizeof(float) * 6 * cn, msg)) ||
        (e = ensure(I, bMgB, sizeof(float) * 72 * cn, msg)) || (e = ensure(I, bMgT, sizeof(float) * 72 * cn, msg)) ||
        (e = ensure(I, bMgZ, sizeof(float) * 72 * cn, msg)) ||
        (e = ensure(I, bMgMinv, sizeof(float) * mgp.minv.size(), msg)) ||
        (e = ensure(I, bMgList, sizeof(int) * std::max<size_t>(mgp.lists.size(), 1), msg)) ||
        (e = ensure(I, bMgNodes, sizeof(int64_t) * std::max<size_t>(mgp.nodes_l.size(), 1), msg)))
      return e;
    DTC_CUDA(cudaMemcpyAsync(I.bufs[bMgDoms], mgp.doms.data(), sizeof(DomDev) * mgp.doms.size(),
                             cudaMemcpyHostToDevice, s));
    if (!mgp.tiles.empty())
      DTC_CUDA(cudaMemcpyAsync(I.bufs[bMgTiles], mgp.tiles.data(), sizeof(Tile) * mgp.tiles.size(),
                               cudaMemcpyHostToDevice, s));
    if (!mgp.svox.empty())
      DTC_CUDA(cudaMemcpyAsync(I.bufs[bMgSvox], mgp.svox.data(), sizeof(float) * mgp.svox.size(),
                               cudaMemcpyHostToDevice, s));
    DTC_CUDA(cudaMemcpyAsync(I.bufs[bMgMinv], mgp.minv.data(), sizeof(float) * mgp.minv.size(),
                             cudaMemcpyHostToDevice, s));
    if (!mgp.lists.empty())
      DTC_CUDA(cudaMemcpyAsync(I.bufs[bMgList], mgp.lists.data(), sizeof(int) * mgp.lists.size(),
                               cudaMemcpyHostToDevice, s));
    if (!mgp.nodes_l.empty())
      DTC_CUDA(cudaMemcpyAsync(I.bufs[bMgNodes], mgp.nodes_l.data(), sizeof(int64_t) * mgp.nodes_l.size(),
                               cudaMemcpyHostToDevice, s));
    DTC_CUDA(cudaMemsetAsync(I.bufs[bMgFlags], 0, cn, s));
    DTC_CUDA(cudaMemsetAsync(I.bufs[bMgBinv32], 0, sizeof(float) * 6 * cn, s));
    DTC_CUDA(cudaMemsetAsync(I.bufs[bMgB], 0, sizeof(float) * 72 * cn, s));
    DTC_CUDA(cudaMemsetAsync(I.bufs[bMgT], 0, sizeof(float) * 72 * cn, s));
    DTC_CUDA(cudaMemsetAsync(I.bufs[bMgZ], 0, sizeof(float) * 72 * cn, s));
    DTC_CUDA(cudaMemsetAsync(I.bufs[bZ32], 0, vbytes32, s));
    DTC_CUDA(cudaMemsetAsync(I.bufs[bT32], 0, vbytes32, s));
    for (int l = 1; l < mgp.nlev; ++l)
      if (mgp.all_n[l] > 0) {
        k_node_setup<8><<<(unsigned)mgp.all_n[l], kThreads, 0, s>>>(
            B<Tile>(I, bMgTiles) + mgp.all_off[l], B<DomDev>(I, bMgDoms) + (size_t)l * ndom, B<float>(I, bMgSvox),
            B<uint8_t>(I, bMgFlags), B<double>(I, bMgDinv64), B<float>(I, bMgDinv32), B<float>(I, bMgBinv32));
        ++L;
      }
    if ((e = launch_check(msg))) return e;
    mgd.P = &mgp;
    mgd.ndom = ndom;
    mgd.tiles = B<Tile>(I, bMgTiles);
    mgd.doms0 = dd;
    mgd.doms = B<DomDev>(I, bMgDoms);
    mgd.svox0 = I.svox();
    mgd.svox = B<float>(I, bMgSvox);
    mgd.binv0 = B<float>(I, bBinv32);
    mgd.binv = B<float>(I, bMgBinv32);
    mgd.minv = B<float>(I, bMgMinv);
    mgd.flags0 = fl;
    mgd.flags = B<uint8_t>(I, bMgFlags);
    mgd.lists = B<int>(I, bMgList);
    mgd.nodes = B<int64_t>(I, bMgNodes);
    mgd.b = B<float>(I, bMgB);
    mgd.t = B<float>(I, bMgT);
    mgd.z = B<float>(I, bMgZ);
    mgd.t0 = B<float>(I, bT32);
    mgd.z0 = B<float>(I, bZ32);
    mgd.nen0 = NEN;
    mgd.bricks0 = W.bi;
    mgd.nbricks0 = W.nbi;
    mgd.nodes0 = W.nodes;
    mgd.nnodes0 = W.nnodes;
    mgd.ke32 = W.ke32;
    mgd.ke20tc = W.ke20tc;
    mgd.err = W.err;
    if (tune) {
      if ((e = autotune_sweep(I, stats_, W, mgd, doms, svox, NEN, msg))) return e;
      if (!I.tensor_matvec) W.ke20tc = mgd.ke20tc = nullptr;   // HEX20: the brick kernel won
      // the timed launches wrote the fine multigrid vectors and the dot accumulators
      DTC_CUDA(cudaMemsetAsync(I.bufs[bZ32], 0, vbytes32, s));
      DTC_CUDA(cudaMemsetAsync(I.bufs[bT32], 0, vbytes32, s));
      DTC_CUDA(cudaMemsetAsync(I.bufs[bZz], 0, sizeof(double) * ncol, s));
      DTC_CUDA(cudaMemsetAsync(I.bufs[bZr], 0, sizeof(double) * ncol, s));
    }
  }

  // the boundary modes (eps = 1e-6, the hard-coded boundary displacement of
  // mod_write_deck.f90:61) and, per column pass, its 24 columns in c_uu
  std::vector<double> modes((size_t)nm * 3 * nl), slices((size_t)ncp * 20 * 3 * kNLC, 0.0);
  macro_modes_of_order(order, 1e-6, modes.data());
  for (int cp = 0; cp < ncp; ++cp)
    for (int lc = 0; lc < kNLC && cp * kNLC + lc < nl; ++lc)
      for (int c = 0; c < 3; ++c)
        for (int l = 0; l < nm; ++l)
          slices[(size_t)cp * 20 * 3 * kNLC + l + nm * c + 3 * nm * lc] = modes[l + nm * c + (size_t)3 * nm * (cp * kNLC + lc)];
  bool want_fields = false;
  for (int d = 0; d < ndom; ++d) want_fields = want_fields || tasks[tidx[d]].out->displ || tasks[tidx[d]].out->force;
  std::vector<ColState> cs(ncol * ncp);
  std::vector<double> hX, hF;
  for (int cp = 0; cp < ncp; ++cp) {
    if (cp > 0) {   // a later column pass starts from zero vectors like the first
      DTC_CUDA(cudaMemsetAsync(I.bufs[bX], 0, vbytes64, s));
      DTC_CUDA(cudaMemsetAsync(I.bufs[bR64], 0, vbytes64, s));
      if (mixed) {
        DTC_CUDA(cudaMemsetAsync(I.bufs[bR32], 0, vbytes32, s));
        DTC_CUDA(cudaMemsetAsync(I.bufs[bX32], 0, vbytes32, s));
        DTC_CUDA(cudaMemsetAsync(I.bufs[bP32], 0, vbytes32, s));
        if (use_mg) {
          DTC_CUDA(cudaMemsetAsync(I.bufs[bZ32], 0, vbytes32, s));
          DTC_CUDA(cudaMemsetAsync(I.bufs[bT32], 0, vbytes32, s));
        }
      }
    }
    DTC_CUDA(cudaMemcpyToSymbolAsync(c_uu, slices.data() + (size_t)cp * 20 * 3 * kNLC, sizeof(double) * 20 * 3 * kNLC,
                                     0, cudaMemcpyHostToDevice, s));
    if (nta) {
      if (order == 2) k_boundary_values<20><<<(unsigned)nta, kThreads, 0, s>>>(ta, dd, fl, X);
      else k_boundary_values<8><<<(unsigned)nta, kThreads, 0, s>>>(ta, dd, fl, X);
      ++L;
    }
    if ((e = launch_check(msg))) return e;
    bool kx_all = false;   // R64 holds K X on every node for the final X (mixed refinement)
    if (!mixed) {
      // b = -(K X)_interior with X = boundary values only (RHS of all 24 load cases, :674-951)
      DTC_CUDA(cudaMemsetAsync(I.bufs[bP64], 0, vbytes64, s));
      DTC_CUDA(cudaMemsetAsync(I.bufs[bW64], 0, vbytes64, s));
      apply_k<double, NEN, false, false>(W, dd, I.svox(), fl, X, R64, -1.0, nullptr, nullptr, s, 1);
      ++L;
      if ((e = run_cg<double, false, NEN>(I, ndom, W, X, R64, B<double>(I, bP64), B<double>(I, bW64), B<double>(I, bDinv64),
                              opt.rtol, nullptr, opt.max_it, L, msg)))
        return e;
      DTC_CUDA(cudaMemcpyAsync(ost, I.bufs[bSt], sizeof(ColState) * ncol, cudaMemcpyDeviceToDevice, s));
    } else {
      // every FP32 work vector starts at zero: the stencil reads boundary and void entries
      if (cp == 0) {
        DTC_CUDA(cudaMemsetAsync(I.bufs[bR32], 0, vbytes32, s));
        DTC_CUDA(cudaMemsetAsync(I.bufs[bX32], 0, vbytes32, s));
        DTC_CUDA(cudaMemsetAsync(I.bufs[bP32], 0, vbytes32, s));
      }
      // inner FP32 solves aim straight at the outer target when FP32 can reach it
      const double inner = opt.inner_rtol > 0 ? opt.inner_rtol : std::max(0.3 * opt.rtol, 1e-7);
      const int max_refine = opt.max_refine > 0 ? opt.max_refine : 12;
      int64_t inner_budget = opt.max_it;
      for (int step = 0; step <= max_refine; ++step) {
        DTC_CUDA(cudaMemsetAsync(I.bufs[bZz], 0, sizeof(double) * ncol, s));
        // from the second check on, K X over every node: its interior part is minus the residual
        // and, once the loop stops (X is final then), it is the reaction force of every node
        kx_all = step > 0 && nta > 0;
        if (kx_all) {
          apply_k<double, NEN, true, false>(W, dd, I.svox(), fl, X, R64, 1.0, nullptr, nullptr, s);
          ++L;
        } else if (nti) {   // first check: X holds the boundary values only, R64 is zero
          apply_k<double, NEN, false, false>(W, dd, I.svox(), fl, X, R64, -1.0, nullptr, nullptr, s, 1);
          ++L;
        }
        if (nti) {
          k_residual_norm<<<gi, kThreads, 0, s>>>(ti, dd, fl, B<double>(I, bDinv64), R64, B<double>(I, bZz));
          ++L;
        }
        k_outer_check<<<ndom, 32, 0, s>>>(ost, B<double>(I, bZz), B<double>(I, bTarget), B<int>(I, bDomAct), opt.rtol,
                                          step == 0);
        k_count_active<<<1, 256, 0, s>>>(B<int>(I, bDomAct), ndom, B<int>(I, bCount));
        L += 2;
        if ((e = launch_check(msg))) return e;
        int h_count = 0;
        DTC_CUDA(cudaMemcpyAsync(&h_count, I.bufs[bCount], sizeof(int), cudaMemcpyDeviceToHost, s));
        DTC_CUDA(cudaStreamSynchronize(s));
        if (h_count == 0 || step == max_refine || inner_budget <= 0) break;
        if (nti) {
          k_start_inner<<<gi, kThreads, 0, s>>>(ti, dd, fl, R64, B<float>(I, bR32), B<float>(I, bX32), B<float>(I, bP32),
                                                ost, kx_all ? -1.0 : 1.0);
          ++L;
        }
        DTC_CUDA(cudaMemsetAsync(I.bufs[bW32], 0, vbytes32, s));
        if (use_mg)
          e = run_cg_mg<NEN>(I, ndom, W, mgd, B<float>(I, bX32), B<float>(I, bR32), B<float>(I, bP32), B<float>(I, bW32),
                        inner, B<double>(I, bTarget), inner_budget, L, msg);
        else if (opt.inner_precond >= 1)
          e = run_cg<float, true, NEN>(I, ndom, W, B<float>(I, bX32), B<float>(I, bR32), B<float>(I, bP32),
                                  B<float>(I, bW32), B<float>(I, bBinv32), inner, B<double>(I, bTarget), inner_budget,
                                  L, msg);
        else
          e = run_cg<float, false, NEN>(I, ndom, W, B<float>(I, bX32), B<float>(I, bR32), B<float>(I, bP32),
                                   B<float>(I, bW32), B<float>(I, bDinv32), inner, B<double>(I, bTarget), inner_budget,
                                   L, msg);
        if (e) return e;
        if (nti) { k_apply_correction<<<gi, kThreads, 0, s>>>(ti, dd, fl, B<float>(I, bX32), X, ost); ++L; }
        k_add_inner_its<<<(unsigned)((ncol + 255) / 256), 256, 0, s>>>(ost, B<ColState>(I, bSt), (int64_t)ncol);
        ++L;
        if ((e = launch_check(msg))) return e;
      }
    }
    // reactions F = K X on all nodes (AA_org * u, :1092-1123) and their projection (ff); the
    // mixed loop's last check already computed them for the final X (readers use active nodes only)
    if (!kx_all) DTC_CUDA(cudaMemsetAsync(R64, 0, vbytes64, s));
    if (nta) {
      if (!kx_all) {
        apply_k<double, NEN, true, false>(W, dd, I.svox(), fl, X, R64, 1.0, nullptr, nullptr, s);
        ++L;
      }
      if (energy) {
        k_energy_gram<<<ga, kThreads, 0, s>>>(ta, dd, fl, X, R64, B<double>(I, bFf), ldg, kNLC * cp, kNLC * cp);
        for (int q = 0; q < cp; ++q) {   // u_q . K u_cp against the kept solutions of earlier passes
          k_energy_gram<<<ga, kThreads, 0, s>>>(ta, dd, fl, B<double>(I, bXkeep) + (size_t)q * (vbytes64 / 8), R64,
                                                B<double>(I, bFf), ldg, kNLC * q, kNLC * cp);
          ++L;
        }
        if (cp + 1 < ncp)
          DTC_CUDA(cudaMemcpyAsync(B<double>(I, bXkeep) + (size_t)cp * (vbytes64 / 8), X, vbytes64,
                                   cudaMemcpyDeviceToDevice, s));
      } else if (order == 2)
        k_project<20><<<ga, kThreads, 0, s>>>(ta, dd, fl, R64, B<double>(I, bFf), cp * kNLC);
      else
        k_project<8><<<ga, kThreads, 0, s>>>(ta, dd, fl, R64, B<double>(I, bFf), 0);
      ++L;
    }
    if ((e = launch_check(msg))) return e;
    DTC_CUDA(cudaMemcpyAsync(cs.data() + ncol * cp, ost, sizeof(ColState) * ncol, cudaMemcpyDeviceToHost, s));
    // optional displacement / force output in reference numbering (load cases of this pass)
    if (want_fields) {
      hX.resize(node_total * 3 * kNLC);
      hF.resize(node_total * 3 * kNLC);
      DTC_CUDA(cudaMemcpyAsync(hX.data(), X, vbytes64, cudaMemcpyDeviceToHost, s));
      DTC_CUDA(cudaMemcpyAsync(hF.data(), R64, vbytes64, cudaMemcpyDeviceToHost, s));
      DTC_CUDA(cudaStreamSynchronize(s));
      for (int d = 0; d < ndom; ++d) {
        dtc_domain_out* o = tasks[tidx[d]].out;
        if (!o->displ && !o->force) continue;
        const MeshPlan& mp = *tasks[tidx[d]].plan;
        const int64_t nn = mp.nn;
        const DomDev& D = doms[d];
        for (int64_t id = 0; id < nn; ++id) {
          const int64_t node = D.node_off + mp.node_grid[id];  // the mesher's grid index is the device node index
          for (int c = 0; c < 3; ++c)
            for (int lc = 0; lc < kNLC && cp * kNLC + lc < nl; ++lc) {
              const size_t src = (size_t)((node * 3 + c) * kNLC + lc);
              const size_t dst = (size_t)(cp * kNLC + lc) * 3 * nn + 3 * id + c;
              if (o->displ) o->displ[dst] = hX[src];
              if (o->force) o->force[dst] = hF[src];
            }
        }
      }
    }
  }
  DTC_CUDA(cudaEventRecord(I.ev_solve[1], s));
  const size_t per_dom = (size_t)std::max(nl * nl, energy ? ldg * ldg : 0);
  std::vector<double> ff(per_dom * ndom);
  DTC_CUDA(cudaMemcpyAsync(ff.data(), I.bufs[bFf], sizeof(double) * ff.size(), cudaMemcpyDeviceToHost, s));
  int h_err = 0;
  DTC_CUDA(cudaMemcpyAsync(&h_err, I.bufs[bErr], sizeof(int), cudaMemcpyDeviceToHost, s));
  DTC_CUDA(cudaStreamSynchronize(s));
  I.flush();
  if (h_err) { msg = "tensor-core matvec: an mbarrier wait timed out"; return DTC_ERR_INTERNAL; }
  stats_.ms_wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  {
    float ms = 0.f;
    DTC_CUDA(cudaEventElapsedTime(&ms, I.ev_solve[0], I.ev_solve[1]));
    stats_.ms_solve = ms;
  }
  for (int d = 0; d < ndom; ++d) {
    DomainTask& t = tasks[tidx[d]];
    dtc_domain_out* o = t.out;
    double* off = order == 2 ? o->macro2->ff : o->ff;
    if (energy) {
      // the Gram blocks below the diagonal pass blocks are the transposes of those above
      std::vector<double> gram((size_t)nl * nl);
      const double* gd = &ff[per_dom * d];
      for (int b = 0; b < nl; ++b)
        for (int a = 0; a < nl; ++a)
          gram[a + (size_t)nl * b] = (a / kNLC <= b / kNLC) ? gd[a + (size_t)ldg * b] : gd[b + (size_t)ldg * a];
      energy_to_ff(order, gram.data(), off);
    } else {
      std::memcpy(off, &ff[per_dom * d], sizeof(double) * nl * nl);
    }
    int64_t* iters = order == 2 ? o->macro2->iters : o->iters;
    double* relres = order == 2 ? o->macro2->relres : o->relres;
    int worst = DTC_DOMAIN_OK;
    int steps = 0;
    for (int j = 0; j < nl; ++j) {
      const ColState& c = cs[ncol * (j / kNLC) + (size_t)d * kNLC + j % kNLC];
      iters[j] = c.its;
      relres[j] = c.dp0 > 0 ? c.dp / c.dp0 : 0.0;
      steps = std::max(steps, (int)c.pad);
      int st = DTC_DOMAIN_OK;
      if (c.reason == kDivergedIts || (mixed && c.active)) st = DTC_DOMAIN_MAX_IT;
      else if (c.reason == kIndefinite) st = DTC_DOMAIN_BREAKDOWN;
      else if (c.reason == kNanOrInf || c.reason == kDivergedDtol) st = DTC_DOMAIN_NONFINITE;
      if (worst == DTC_DOMAIN_OK) worst = st;
      stats_.dof_iterations += (double)t.plan->n_free_dof * (double)c.its;
    }
    o->refine_steps = mixed ? steps : 0;
    o->status = worst;
  }
  if (keep != kKeepNone) {
    DeviceSolver::Impl::AdjChunk c;
    c.doms = doms;
    for (int d = 0; d < ndom; ++d) c.index.push_back(tasks[tidx[d]].index);
    c.nodes = node_total;
    c.voxels = (int64_t)svox.size();
    c.on_device = keep == kKeepDevice;
    if (!c.on_device) {
      c.X.resize((size_t)node_total * 72);
      c.svox = svox;
      DTC_CUDA(cudaMemcpyAsync(c.X.data(), X, vbytes64, cudaMemcpyDeviceToHost, s));
      DTC_CUDA(cudaStreamSynchronize(s));
    }
    I.adj.push_back(std::move(c));
    I.adj_nen = NEN;
  }
  return DTC_OK;
}

int DeviceSolver::prepare(std::vector<DomainTask>& tasks, const dtc_options& opt, double nu, HostBatchPtr& out,
                          std::string& msg) {
  int nen = 0;
  for (const DomainTask& t : tasks) {
    if (t.plan->status != DTC_DOMAIN_OK) continue;
    if (nen && t.in->elem_type != nen) { msg = "all domains of one solve must share the element type"; return DTC_ERR_INVALID_ARGUMENT; }
    nen = t.in->elem_type;
  }
  out.reset(new (std::nothrow) HostBatch());
  if (!out) return DTC_ERR_OUT_OF_MEMORY;
  out->nen = nen;
  if (nen == 0) return DTC_OK;
  return nen == 20 ? prepare_nen<20>(tasks, opt, nu, *out) : prepare_nen<8>(tasks, opt, nu, *out);
}

int DeviceSolver::solve(std::vector<DomainTask>& tasks, const dtc_options& opt, double nu, HostBatchPtr batch,
                        std::string& msg) {
  if (!batch || batch->nen == 0) return DTC_OK;
  DTC_CUDA(cudaSetDevice(impl_->device));
  impl_->adj_nu = nu;
  return batch->nen == 20 ? solve_nen<20>(*impl_, stats_, tasks, opt, nu, keep_, *batch, msg)
                          : solve_nen<8>(*impl_, stats_, tasks, opt, nu, keep_, *batch, msg);
}

int DeviceSolver::solve(std::vector<DomainTask>& tasks, const dtc_options& opt, double nu, std::string& msg) {
  HostBatchPtr batch;
  if (int e = prepare(tasks, opt, nu, batch, msg)) return e;
  return solve(tasks, opt, nu, std::move(batch), msg);
}

int DeviceSolver::upload_voxels(HostBatch* hb, std::string& msg) {
  if (!hb || hb->nen == 0 || hb->svox.empty()) return DTC_OK;
  Impl& I = *impl_;
  auto stage = [&]() -> int {
    DTC_CUDA(cudaSetDevice(I.device));
    if (!I.up_stream) {
      DTC_CUDA(cudaStreamCreateWithFlags(&I.up_stream, cudaStreamNonBlocking));
      DTC_CUDA(cudaEventCreateWithFlags(&I.up_ev[0], cudaEventDisableTiming));
      DTC_CUDA(cudaEventCreateWithFlags(&I.up_ev[1], cudaEventDisableTiming));
    }
    const int k = I.up_next;
    const size_t n = hb->svox.size();
    // the slot's last reader, the pass before the one now solving, has finished; its copy too
    DTC_CUDA(cudaEventSynchronize(I.up_ev[k]));
    if (I.up_cap[k] < n) {
      if (I.up_pin[k]) cudaFreeHost(I.up_pin[k]);
      if (I.up_dev[k]) cudaFree(I.up_dev[k]);
      I.up_pin[k] = nullptr;
      I.up_dev[k] = nullptr;
      I.up_cap[k] = 0;
      DTC_CUDA(cudaMallocHost(&I.up_pin[k], sizeof(float) * n));
      DTC_CUDA(cudaMalloc(&I.up_dev[k], sizeof(float) * n));
      I.up_cap[k] = n;
    }
    std::memcpy(I.up_pin[k], hb->svox.data(), sizeof(float) * n);
    DTC_CUDA(cudaMemcpyAsync(I.up_dev[k], I.up_pin[k], sizeof(float) * n, cudaMemcpyHostToDevice, I.up_stream));
    DTC_CUDA(cudaEventRecord(I.up_ev[k], I.up_stream));
    hb->up_slot = k;
    I.up_next = 1 - k;
    return DTC_OK;
  };
  const int rc = stage();
  // a failed allocation leaves a (non-sticky) last error behind: clear it, so that the next
  // launch check does not report it for a kernel
  if (rc != DTC_OK) cudaGetLastError();
  return rc;
}

void DeviceSolver::clear_kept() {
  if (impl_) impl_->adj.clear();
}

namespace {

// Nodal mixes of the kept load-case displacements: V[node][c][b] = sum_a X[node][c][a] G[a][b],
// b < 6 (the columns of dL/dff the 6x6 tensor depends on).  One thread per (node, c).
__global__ void k_adj_mix(const int64_t* __restrict__ blocks, const DomDev* __restrict__ doms,
                          const double* __restrict__ X, const double* __restrict__ G, double* __restrict__ V) {
  const int64_t e = blocks[2 * blockIdx.x], start = blocks[2 * blockIdx.x + 1];
  const DomDev D = doms[e];
  const int64_t nn = (int64_t)D.n[0] * D.n[1] * D.n[2];
  const int64_t i = start + threadIdx.x;
  if (i >= 3 * nn) return;
  const int64_t node = D.node_off + i / 3;
  const int c = (int)(i % 3);
  const double* x = X + vec_index(node, c, 0);
  const double* g = G + (int64_t)e * kNLC * 6;
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int a = 0; a < kNLC; ++a) {
    const double xa = x[a];
#pragma unroll
    for (int b = 0; b < 6; ++b) v[b] = fma(xa, g[a * 6 + b], v[b]);
  }
#pragma unroll
  for (int b = 0; b < 6; ++b) V[(node * 3 + c) * 8 + b] = v[b];
}

// dL/dE_v = a * sum_{b<6} V_b,v^T Khat u_b,v for every kept voxel (0 elsewhere): the
// derivative of the energy products u_a^T K u_b (self-adjoint operator, so no adjoint solve).
__global__ void k_energy_grad(const int64_t* __restrict__ blocks, const DomDev* __restrict__ doms,
                              const float* __restrict__ svox, const double* __restrict__ X,
                              const double* __restrict__ V, float* __restrict__ grad) {
  const int64_t e = blocks[2 * blockIdx.x], start = blocks[2 * blockIdx.x + 1];
  const DomDev D = doms[e];
  const int64_t nvox = (int64_t)D.L[0] * D.L[1] * D.L[2];
  const int64_t v = start + threadIdx.x;
  if (v >= nvox) return;
  const int64_t gi = D.vox_off + v;
  if (svox[gi] == 0.0f) { grad[gi] = 0.0f; return; }
  const int vx = (int)(v % D.L[0]), vy = (int)((v / D.L[0]) % D.L[1]), vz = (int)(v / ((int64_t)D.L[0] * D.L[1]));
  int64_t nodes[8];
#pragma unroll
  for (int a = 0; a < 8; ++a)
    nodes[a] = node_index(D, vx + Elem<8>::off(a, 0), vy + Elem<8>::off(a, 1), vz + Elem<8>::off(a, 2));
  double sum = 0.0;
  for (int b = 0; b < 6; ++b) {
    double u[24], w[24];
#pragma unroll
    for (int a = 0; a < 8; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        u[3 * a + c] = X[vec_index(nodes[a], c, b)];
        w[3 * a + c] = V[(nodes[a] * 3 + c) * 8 + b];
      }
#pragma unroll
    for (int i = 0; i < 24; ++i) {
      double r = 0.0;
#pragma unroll
      for (int j = 0; j < 24; ++j) r = fma(c_khat64[i + 24 * j], u[j], r);
      sum = fma(w[i], r, sum);
    }
  }
  grad[gi] = (float)(D.scale * sum);
}

// dL/dff (24 x 24, column-major) of L through C = fv * meps (mod_struct_calcmat.f90:345-359,
// 434-439) given dL/dC (column-major 6 x 6): only the first 6 load-case columns are touched.
void dloss_dff(const double* dc, const int64_t L[3], const double delta, double* lff) {
  std::memset(lff, 0, sizeof(double) * 576);
  const double X = (double)L[0] * delta, Y = (double)L[1] * delta, Z = (double)L[2] * delta;
  const double meps[6] = {1e6, 1e6, 1e6, -1e6, -1e6, 1e6};
  auto add = [&](int r, int c, double w) { lff[(r - 1) + 24 * c] += w; };
  for (int c = 0; c < 6; ++c) {
    const double g0 = dc[0 + 6 * c] * meps[c], g1 = dc[1 + 6 * c] * meps[c], g2 = dc[2 + 6 * c] * meps[c];
    const double g3 = dc[3 + 6 * c] * meps[c], g4 = dc[4 + 6 * c] * meps[c], g5 = dc[5 + 6 * c] * meps[c];
    for (int r : {2, 3, 6, 7}) add(r, c, g0 / (Y * Z));
    for (int r : {11, 12, 15, 16}) add(r, c, g1 / (X * Z));
    for (int r : {21, 22, 23, 24}) add(r, c, g2 / (X * Y));
    for (int r : {3, 4, 7, 8}) add(r, c, 0.5 * g3 / (X * Z));
    for (int r : {10, 11, 14, 15}) add(r, c, 0.5 * g3 / (Y * Z));
    for (int r : {5, 6, 7, 8}) add(r, c, 0.5 * g4 / (X * Y));
    for (int r : {18, 19, 22, 23}) add(r, c, 0.5 * g4 / (Y * Z));
    for (int r : {13, 14, 15, 16}) add(r, c, 0.5 * g5 / (X * Y));
    for (int r : {19, 20, 23, 24}) add(r, c, 0.5 * g5 / (X * Z));
  }
}

}  // namespace

int DeviceSolver::energy_grad(const double* dloss_dc, float* const* grad_e, int64_t n, bool grad_on_device,
                              std::string& msg) {
  Impl& I = *impl_;
  DTC_CUDA(cudaSetDevice(I.device));
  cudaStream_t s = I.stream;
  if (I.adj.empty()) { msg = "energy_grad: no kept displacements (solve with keep_displacements = 1 first)"; return DTC_ERR_INVALID_ARGUMENT; }
  if (I.adj_nen != 8) { msg = "energy_grad: HEX08 domains only"; return DTC_ERR_INVALID_ARGUMENT; }
  // G = vv_bc^-1 dL/dff (24 x 6 per domain, row-major a * 6 + b): the energy-product form of ff
  double uu[8 * 3 * 24], vinv[576];
  macro_modes(1e-6, uu);
  for (int lc = 0; lc < 24; ++lc)
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < 8; ++l) vinv[(8 * k + l) + 24 * lc] = uu[l + 8 * k + 24 * lc];
  {
    // Gauss-Jordan on a copy (the same inverse the forward uses)
    double a[576], inv[576];
    std::memcpy(a, vinv, sizeof(a));
    for (int i = 0; i < 576; ++i) inv[i] = (i % 25 == 0) ? 1.0 : 0.0;
    for (int c = 0; c < 24; ++c) {
      int p = c;
      for (int r = c + 1; r < 24; ++r) if (std::fabs(a[r + 24 * c]) > std::fabs(a[p + 24 * c])) p = r;
      for (int k = 0; k < 24; ++k) { std::swap(a[c + 24 * k], a[p + 24 * k]); std::swap(inv[c + 24 * k], inv[p + 24 * k]); }
      const double d = a[c + 24 * c];
      for (int k = 0; k < 24; ++k) { a[c + 24 * k] /= d; inv[c + 24 * k] /= d; }
      for (int r = 0; r < 24; ++r) {
        if (r == c) continue;
        const double f = a[r + 24 * c];
        if (f == 0.0) continue;
        for (int k = 0; k < 24; ++k) { a[r + 24 * k] -= f * a[c + 24 * k]; inv[r + 24 * k] -= f * inv[c + 24 * k]; }
      }
    }
    std::memcpy(vinv, inv, sizeof(inv));
  }
  int e;
  for (const Impl::AdjChunk& ch : I.adj) {
    const int nd = (int)ch.doms.size();
    std::vector<double> G((size_t)nd * kNLC * 6, 0.0);
    for (int d = 0; d < nd; ++d) {
      const int64_t k = ch.index[d];
      if (k < 0 || k >= n) continue;
      const DomDev& D = ch.doms[d];
      const int64_t L[3] = {D.L[0], D.L[1], D.L[2]};
      double lff[576];
      dloss_dff(dloss_dc + 36 * k, L, D.delta, lff);
      for (int a = 0; a < 24; ++a)
        for (int b = 0; b < 6; ++b) {
          double sum = 0.0;
          for (int r = 0; r < 24; ++r) sum += vinv[a + 24 * r] * lff[r + 24 * b];
          G[(size_t)d * kNLC * 6 + a * 6 + b] = sum;
        }
    }
    // block tables (domain, first item) for the node and voxel kernels
    std::vector<int64_t> nb, vb;
    for (int d = 0; d < nd; ++d) {
      const DomDev& D = ch.doms[d];
      const int64_t items = 3 * (int64_t)D.n[0] * D.n[1] * D.n[2], vox = (int64_t)D.L[0] * D.L[1] * D.L[2];
      for (int64_t q = 0; q < items; q += 256) { nb.push_back(d); nb.push_back(q); }
      for (int64_t q = 0; q < vox; q += 128) { vb.push_back(d); vb.push_back(q); }
    }
    if ((e = ensure(I, bAdjG, sizeof(double) * G.size(), msg)) ||
        (e = ensure(I, bAdjV, sizeof(double) * 24 * std::max<int64_t>(ch.nodes, 1), msg)) ||
        (e = ensure(I, bAdjBlk, sizeof(int64_t) * (nb.size() + vb.size()), msg)) ||
        (e = ensure(I, bAdjGrad, sizeof(float) * std::max<int64_t>(ch.voxels, 1), msg)) ||
        (e = ensure(I, bAdjDoms, sizeof(DomDev) * nd, msg)))
      return e;
    const double* X;
    const float* sv;
    if (ch.on_device) {
      X = B<double>(I, bX);
      sv = I.svox();
    } else {
      if ((e = ensure(I, bAdjX, sizeof(double) * ch.X.size(), msg)) ||
          (e = ensure(I, bAdjSvox, sizeof(float) * std::max<size_t>(ch.svox.size(), 1), msg)))
        return e;
      DTC_CUDA(cudaMemcpyAsync(I.bufs[bAdjX], ch.X.data(), sizeof(double) * ch.X.size(), cudaMemcpyHostToDevice, s));
      DTC_CUDA(cudaMemcpyAsync(I.bufs[bAdjSvox], ch.svox.data(), sizeof(float) * ch.svox.size(),
                               cudaMemcpyHostToDevice, s));
      X = B<double>(I, bAdjX);
      sv = B<float>(I, bAdjSvox);
    }
    DTC_CUDA(cudaMemcpyAsync(I.bufs[bAdjG], G.data(), sizeof(double) * G.size(), cudaMemcpyHostToDevice, s));
    DTC_CUDA(cudaMemcpyAsync(I.bufs[bAdjDoms], ch.doms.data(), sizeof(DomDev) * nd, cudaMemcpyHostToDevice, s));
    std::vector<int64_t> blk(nb);
    blk.insert(blk.end(), vb.begin(), vb.end());
    DTC_CUDA(cudaMemcpyAsync(I.bufs[bAdjBlk], blk.data(), sizeof(int64_t) * blk.size(), cudaMemcpyHostToDevice, s));
    const int64_t* blocks = B<int64_t>(I, bAdjBlk);
    if (!nb.empty())
      k_adj_mix<<<(unsigned)(nb.size() / 2), 256, 0, s>>>(blocks, B<DomDev>(I, bAdjDoms), X, B<double>(I, bAdjG),
                                                          B<double>(I, bAdjV));
    if (!vb.empty())
      k_energy_grad<<<(unsigned)(vb.size() / 2), 128, 0, s>>>(blocks + nb.size(), B<DomDev>(I, bAdjDoms), sv, X,
                                                              B<double>(I, bAdjV), B<float>(I, bAdjGrad));
    if ((e = launch_check(msg))) return e;
    if (grad_on_device) {
      for (int d = 0; d < nd; ++d) {
        const int64_t k = ch.index[d];
        if (k < 0 || k >= n || !grad_e[k]) continue;
        const DomDev& D = ch.doms[d];
        DTC_CUDA(cudaMemcpyAsync(grad_e[k], B<float>(I, bAdjGrad) + D.vox_off,
                                 sizeof(float) * (size_t)D.L[0] * D.L[1] * D.L[2], cudaMemcpyDeviceToDevice, s));
      }
      DTC_CUDA(cudaStreamSynchronize(s));
      continue;
    }
    std::vector<float> hg((size_t)ch.voxels);
    if (ch.voxels)
      DTC_CUDA(cudaMemcpyAsync(hg.data(), I.bufs[bAdjGrad], sizeof(float) * hg.size(), cudaMemcpyDeviceToHost, s));
    DTC_CUDA(cudaStreamSynchronize(s));
    for (int d = 0; d < nd; ++d) {
      const int64_t k = ch.index[d];
      if (k < 0 || k >= n || !grad_e[k]) continue;
      const DomDev& D = ch.doms[d];
      std::memcpy(grad_e[k], hg.data() + D.vox_off, sizeof(float) * (size_t)D.L[0] * D.L[1] * D.L[2]);
    }
  }
  return DTC_OK;
}

}  // namespace dtc
