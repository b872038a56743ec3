// mg.cuh -- multigrid V-cycle that preconditions the FP32 inner solve (HEX08 grids; a HEX20
// fine level is first coarsened to the HEX08 mesh of the same voxels).
//
// Not a step of the reference (its KSP uses PCJACOBI, f-src/mod_dtc_main_subroutines.f90:
// 995-1078); it only changes how fast the inner FP32 solve of the iterative refinement
// reaches its tolerance, never the FP64 outer residual or the tensor it converges to.
//
// Hierarchy: level l+1 halves the voxel grid of level l (ceil(L/2) voxels per edge); a coarse
// voxel carries the mean of the moduli of its <= 8 children (void and missing children count
// as 0) and twice the edge, so its element matrix is 2 * mean(E) * a * Khat.  For moduli that
// are constant inside each coarse voxel this equals the Galerkin product P^T K P of the
// trilinear prolongation P, because the coarse trilinear space is nested in the fine one.
// Every level keeps all nodes on its domain box fixed (zero correction).  The coarsest level
// (at most 4 voxels per edge, at most 27 interior nodes) is solved with a dense inverse.
//
// Smoother: one damped node-block-Jacobi sweep x = omega D^-1 r, D the 3x3 diagonal blocks
// (Chebyshev of degree 1 on [lambda*/30, 1.1 lambda*]; lambda* = the largest eigenvalue of
// Khat v = lambda De v for the unit voxel, De its node-block diagonal, bounds
// lambda_max(D^-1 K) for any assembly of scaled voxels), the same before and after the coarse
// correction, so the V-cycle is a fixed SPD operator.
//
// One V-cycle per CG iteration, per level l that is not a domain's coarsest:
//   t_l = omega D_l^-1 b_l                        k_mg_jacobi_flat (fine level: k_update_flat)
//   r_l = b_l - K_l t_l                           k_mg_matvec<kMgRes>
//   b_{l+1} = P^T r_l                             k_mg_restrict_flat
//   (level l+1: recurse, or z_{l+1} = K^-1 b)     ...  / k_mg_coarse
//   t_l += P z_{l+1}                              k_mg_prolong_flat
//   z_l = t_l + omega D_l^-1 (b_l - K_l t_l)      k_mg_matvec<kMgPost> (+ z.z, z.b on level 0)
// Levels >= 2 apply the smoothing step twice before and twice after the coarse correction.
#pragma once

namespace dtc {

constexpr int kMgMaxCoarse = 4;                  // voxels per edge on the coarsest level
constexpr int kMgDenseN = 81;                    // 3 * 3^3 interior DOFs at most
enum { kMgRes = 0, kMgPost = 1 };
// node-list entries: (domain << kListShift) | node
constexpr int kListShift = 40;
constexpr int64_t kListNodeMask = (int64_t(1) << kListShift) - 1;

// Residual / smoother on one level's interior tiles (the slab sweep of k_matvec).
//   kMgRes : y = b - K u
//   kMgPost: y = u + omega D^-1 (b - K u);  DOT: zz += y.y, zr += y.b per (domain, load case)
// MINB: CTAs per SM the register allocation is sized for (6: at most 80 registers; 8: 64);
// xlen: nodes per row of the tile list (kSweepX)
template <int MODE, bool DOT, int MINB = 6>
__global__ void __launch_bounds__(kThreads, MINB) k_mg_matvec(const Tile* __restrict__ tiles, const DomDev* __restrict__ doms,
                                                        const float* __restrict__ svox,
                                                        const float* __restrict__ binv, const float* __restrict__ b,
                                                        const float* __restrict__ u, float* __restrict__ y, float omega,
                                                        double* __restrict__ acc_zz, double* __restrict__ acc_zr,
                                                        const int* __restrict__ dom_active, int xlen) {
  __shared__ double red[32];
  const Tile t = tiles[blockIdx.x / 3];
  if (dom_active && !dom_active[t.dom]) return;
  const DomDev D = doms[t.dom];
  const int lc = (blockIdx.x % 3) * kLcGroup + (threadIdx.x & 7);
  const int row = threadIdx.x >> 3;
  const int yy = t.y0 + (row & 3), zz = t.z0 + (row >> 2);
  double szz = 0.0, szr = 0.0;
  if (yy >= 1 && yy <= D.n[1] - 2 && zz >= 1 && zz <= D.n[2] - 2) {
    const int sy = D.n[0] * (3 * kNLC), sz = D.n[0] * D.n[1] * (3 * kNLC);
    const float* rp = u + vec_index(node_index(D, t.x0 - 1, yy, zz), 0, lc);   // plane x0 - 1
    VoxRow V;
    float sv[2][2];
    float cur[3] = {0.f, 0.f, 0.f}, nxt[3] = {0.f, 0.f, 0.f};
    V.start(svox, D, t.x0 - 1, yy, zz);
    V.load(sv);
    bool anyp = (sv[0][0] != 0.f) | (sv[0][1] != 0.f) | (sv[1][0] != 0.f) | (sv[1][1] != 0.f);
    row_slab<true>(rp, sy, sz, sv, cur, nxt);
    const int xe = min(D.n[0] - 2, t.x0 + xlen - 1);
#pragma unroll 1
    for (int x = t.x0; x <= xe; ++x) {
      rp += 3 * kNLC;   // plane x
      ++V.p;
      V.load(sv);
      const bool anyc = (sv[0][0] != 0.f) | (sv[0][1] != 0.f) | (sv[1][0] != 0.f) | (sv[1][1] != 0.f);
#pragma unroll
      for (int c = 0; c < 3; ++c) { cur[c] = nxt[c]; nxt[c] = 0.f; }
      row_slab<false>(rp, sy, sz, sv, cur, nxt);
      if (anyp | anyc) {
        const int64_t k0 = rp - u;
        float res[3], bc[3], v[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          bc[c] = b[k0 + c * kNLC];
          res[c] = bc[c] - (float)(D.scale * (double)cur[c]);
        }
        if (MODE == kMgRes) {
#pragma unroll
          for (int c = 0; c < 3; ++c) v[c] = res[c];
        } else {
          float dz[3];
          block_jacobi(binv, node_index(D, x, yy, zz), omega, res, dz);
#pragma unroll
          for (int c = 0; c < 3; ++c) v[c] = __ldg(rp + c * kNLC) + dz[c];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          y[k0 + c * kNLC] = v[c];
          if (DOT) {
            szz += (double)v[c] * (double)v[c];
            szr += (double)v[c] * (double)bc[c];
          }
        }
      }
      anyp = anyc;
    }
  }
  if (DOT) {
    const int64_t col = (int64_t)t.dom * kNLC + lc;
    const double s1 = block_sum_lc<double>(szz, red);
    __syncthreads();
    const double s2 = block_sum_lc<double>(szr, red);
    if (threadIdx.x < 8) {
      atomicAdd(acc_zz + col, s1);
      atomicAdd(acc_zr + col, s2);
    }
  }
}

// Node-local second half of the residual / smoother when K t was applied by the brick kernel
// (HEX20 fine level), z holding -K t on entry:
//   kMgRes : z = b + z
//   kMgPost: z = t + omega D^-1 (b + z);  DOT: zz += z.z, zr += z.b
template <int MODE, bool DOT>
__global__ void __launch_bounds__(kThreads) k_mg_combine(const Tile* __restrict__ tiles, const DomDev* __restrict__ doms,
                                                         const uint8_t* __restrict__ flags,
                                                         const float* __restrict__ binv, const float* __restrict__ b,
                                                         const float* __restrict__ t_in, float* __restrict__ z,
                                                         float omega, double* __restrict__ acc_zz,
                                                         double* __restrict__ acc_zr,
                                                         const int* __restrict__ dom_active) {
  __shared__ double red[32];
  const Tile t = tiles[blockIdx.x / 3];
  if (dom_active && !dom_active[t.dom]) return;
  const DomDev D = doms[t.dom];
  const int lc = (blockIdx.x % 3) * kLcGroup + (threadIdx.x & 7);
  const int row = threadIdx.x >> 3;
  const int yy = t.y0 + (row & 3), zz = t.z0 + (row >> 2);
  double szz = 0.0, szr = 0.0;
  if (yy >= 1 && yy <= D.n[1] - 2 && zz >= 1 && zz <= D.n[2] - 2) {
    for (int i = 0; i < kTileX; ++i) {
      const int x = t.x0 + i;
      if (x > D.n[0] - 2) break;
      const int64_t n = node_index(D, x, yy, zz);
      if (!(flags[n] & kNodeActive)) continue;
      const int64_t k0 = vec_index(n, 0, lc);
      float bc[3], res[3], v[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        bc[c] = b[k0 + c * kNLC];
        res[c] = bc[c] + z[k0 + c * kNLC];
      }
      if (MODE == kMgRes) {
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = res[c];
      } else {
        float dz[3];
        block_jacobi(binv, n, omega, res, dz);
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = t_in[k0 + c * kNLC] + dz[c];
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        z[k0 + c * kNLC] = v[c];
        if (DOT) {
          szz += (double)v[c] * (double)v[c];
          szr += (double)v[c] * (double)bc[c];
        }
      }
    }
  }
  if (DOT) {
    const int64_t col = (int64_t)t.dom * kNLC + lc;
    const double s1 = block_sum_lc<double>(szz, red);
    __syncthreads();
    const double s2 = block_sum_lc<double>(szr, red);
    if (threadIdx.x < 8) {
      atomicAdd(acc_zz + col, s1);
      atomicAdd(acc_zr + col, s2);
    }
  }
}

// -------------------------------------------------------------------------------------
// Grid transfers over node lists: one thread per (active interior node, 4 load cases) with
// 16-byte loads and stores, all threads independent.  (A tile walk, one thread per node row and
// load case, visits a tile's nodes one after the other including its inactive ones, and ran at
// 27-38 % of the HBM bandwidth; these lists carry only the active nodes.)
constexpr int kQuads = kNLC / 4;

__device__ __forceinline__ float4 ldq(const float* p) { return __ldg(reinterpret_cast<const float4*>(p)); }
__device__ __forceinline__ void fmaq(float w, float4 v, float4& s) {
  s.x = fmaf(w, v.x, s.x);
  s.y = fmaf(w, v.y, s.y);
  s.z = fmaf(w, v.z, s.z);
  s.w = fmaf(w, v.w, s.w);
}

// t_f += P z_c (trilinear) over a fine level's node list; domains without a coarser level
// (their coarse record is empty) are skipped.
__global__ void __launch_bounds__(256) k_mg_prolong_flat(const int64_t* __restrict__ list, int64_t nitems,
                                                         const DomDev* __restrict__ doms_f,
                                                         const DomDev* __restrict__ doms_c,
                                                         const float* __restrict__ z_c, float* __restrict__ t_f,
                                                         const int* __restrict__ dom_active) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nitems) return;
  const int64_t e = __ldg(list + i / kQuads);
  const int dom = (int)(e >> kListShift);
  if (dom_active && !dom_active[dom]) return;
  const DomDev C = doms_c[dom];
  if (C.n[0] == 0) return;
  const DomDev F = doms_f[dom];
  const int64_t nf = e & kListNodeMask;
  const int loc = (int)(nf - F.node_off);
  const int x = loc % F.n[0], yz = loc / F.n[0];
  const int y = yz % F.n[1], z = yz / F.n[1];
  const int lc0 = 4 * (int)(i % kQuads);
  const int cx0 = x >> 1, cx1 = (x + 1) >> 1, cy0 = y >> 1, cy1 = (y + 1) >> 1, cz0 = z >> 1, cz1 = (z + 1) >> 1;
  float4 s[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) s[c] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int kz = 0; kz < 2; ++kz)
#pragma unroll
    for (int ky = 0; ky < 2; ++ky)
#pragma unroll
      for (int kx = 0; kx < 2; ++kx) {
        const int64_t k = vec_index(node_index(C, kx ? cx1 : cx0, ky ? cy1 : cy0, kz ? cz1 : cz0), 0, lc0);
#pragma unroll
        for (int c = 0; c < 3; ++c) fmaq(0.125f, ldq(z_c + k + c * kNLC), s[c]);
      }
  const int64_t k0 = vec_index(nf, 0, lc0);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float4* q = reinterpret_cast<float4*>(t_f + k0 + c * kNLC);
    float4 v = *q;
    v.x += s[c].x;
    v.y += s[c].y;
    v.z += s[c].z;
    v.w += s[c].w;
    *q = v;
  }
}

// b_c = P^T r_f (full weighting) over a coarse level's node list.
__global__ void __launch_bounds__(256) k_mg_restrict_flat(const int64_t* __restrict__ list, int64_t nitems,
                                                          const DomDev* __restrict__ doms_c,
                                                          const DomDev* __restrict__ doms_f,
                                                          const float* __restrict__ r_f, float* __restrict__ b_c,
                                                          const int* __restrict__ dom_active) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nitems) return;
  const int64_t e = __ldg(list + i / kQuads);
  const int dom = (int)(e >> kListShift);
  if (dom_active && !dom_active[dom]) return;
  const DomDev C = doms_c[dom];
  const DomDev F = doms_f[dom];
  const int64_t nc = e & kListNodeMask;
  const int loc = (int)(nc - C.node_off);
  const int x = loc % C.n[0], yz = loc / C.n[0];
  const int y = yz % C.n[1], z = yz / C.n[1];
  const int lc0 = 4 * (int)(i % kQuads);
  float4 s[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) s[c] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int dz = -1; dz <= 1; ++dz) {
    const int fz = 2 * z + dz;
    if (fz > F.n[2] - 1) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int fy = 2 * y + dy;
      if (fy > F.n[1] - 1) continue;
#pragma unroll
      for (int dx = -1; dx <= 1; ++dx) {
        const int fx = 2 * x + dx;
        if (fx > F.n[0] - 1) continue;
        const float wgt = (dx ? 0.5f : 1.f) * (dy ? 0.5f : 1.f) * (dz ? 0.5f : 1.f);
        const int64_t k = vec_index(node_index(F, fx, fy, fz), 0, lc0);
#pragma unroll
        for (int c = 0; c < 3; ++c) fmaq(wgt, ldq(r_f + k + c * kNLC), s[c]);
      }
    }
  }
  const int64_t k0 = vec_index(nc, 0, lc0);
#pragma unroll
  for (int c = 0; c < 3; ++c) *reinterpret_cast<float4*>(b_c + k0 + c * kNLC) = s[c];
}

// t = omega D^-1 b (pre-smoothing from a zero guess) over a level's node list, for the domains
// that have a coarser level (the record of the next level is not empty).
__global__ void __launch_bounds__(256) k_mg_jacobi_flat(const int64_t* __restrict__ list, int64_t nitems,
                                                        const DomDev* __restrict__ doms_next,
                                                        const float* __restrict__ binv, const float* __restrict__ b,
                                                        float omega, float* __restrict__ t_out,
                                                        const int* __restrict__ dom_active) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nitems) return;
  const int64_t e = __ldg(list + i / kQuads);
  const int dom = (int)(e >> kListShift);
  if (dom_active && !dom_active[dom]) return;
  if (doms_next[dom].n[0] == 0) return;
  const int64_t n = e & kListNodeMask;
  const int64_t k0 = vec_index(n, 0, 4 * (int)(i % kQuads));
  const float4 r0 = ldq(b + k0), r1 = ldq(b + k0 + kNLC), r2 = ldq(b + k0 + 2 * kNLC);
  const float* bp = binv + n * 6;
  const float b0 = __ldg(bp), b1 = __ldg(bp + 1), b2 = __ldg(bp + 2), b3 = __ldg(bp + 3), b4 = __ldg(bp + 4),
              b5 = __ldg(bp + 5);
  float4 z0, z1, z2;
  z0.x = omega * (b0 * r0.x + b3 * r1.x + b4 * r2.x);
  z1.x = omega * (b3 * r0.x + b1 * r1.x + b5 * r2.x);
  z2.x = omega * (b4 * r0.x + b5 * r1.x + b2 * r2.x);
  z0.y = omega * (b0 * r0.y + b3 * r1.y + b4 * r2.y);
  z1.y = omega * (b3 * r0.y + b1 * r1.y + b5 * r2.y);
  z2.y = omega * (b4 * r0.y + b5 * r1.y + b2 * r2.y);
  z0.z = omega * (b0 * r0.z + b3 * r1.z + b4 * r2.z);
  z1.z = omega * (b3 * r0.z + b1 * r1.z + b5 * r2.z);
  z2.z = omega * (b4 * r0.z + b5 * r1.z + b2 * r2.z);
  z0.w = omega * (b0 * r0.w + b3 * r1.w + b4 * r2.w);
  z1.w = omega * (b3 * r0.w + b1 * r1.w + b5 * r2.w);
  z2.w = omega * (b4 * r0.w + b5 * r1.w + b2 * r2.w);
  *reinterpret_cast<float4*>(t_out + k0) = z0;
  *reinterpret_cast<float4*>(t_out + k0 + kNLC) = z1;
  *reinterpret_cast<float4*>(t_out + k0 + 2 * kNLC) = z2;
}

// Coarsest level: z = Minv b over the <= 27 interior nodes of each listed domain (one CTA per
// domain, Minv 81 x 81 row-major on the DOFs 3 * ((x-1) + 3 (y-1) + 9 (z-1)) + c).
// DOT (the coarsest level is the finest one): zz += z.z, zr += z.b.
template <bool DOT>
__global__ void __launch_bounds__(256) k_mg_coarse(const int* __restrict__ list, const DomDev* __restrict__ doms,
                                                   const float* __restrict__ minv, const float* __restrict__ b,
                                                   float* __restrict__ z, double* __restrict__ acc_zz,
                                                   double* __restrict__ acc_zr, const int* __restrict__ dom_active) {
  __shared__ float sb[kMgDenseN * kNLC];
  __shared__ double red[2][kNLC];
  const int d = list[blockIdx.x];
  if (dom_active && !dom_active[d]) return;
  const DomDev D = doms[d];
  const int ix = D.n[0] - 2, iy = D.n[1] - 2, iz = D.n[2] - 2;   // interior nodes per axis (<= 3)
  for (int i = threadIdx.x; i < kMgDenseN * kNLC; i += blockDim.x) {
    const int lc = i % kNLC, dof = i / kNLC, node = dof / 3, c = dof % 3;
    const int x = node % 3, y = (node / 3) % 3, zc = node / 9;
    float v = 0.f;
    if (x < ix && y < iy && zc < iz) v = b[vec_index(node_index(D, x + 1, y + 1, zc + 1), c, lc)];
    sb[i] = v;
  }
  if (threadIdx.x < 2 * kNLC) red[threadIdx.x / kNLC][threadIdx.x % kNLC] = 0.0;
  __syncthreads();
  const float* M = minv + (int64_t)d * kMgDenseN * kMgDenseN;
  for (int i = threadIdx.x; i < kMgDenseN * kNLC; i += blockDim.x) {
    const int lc = i % kNLC, dof = i / kNLC, node = dof / 3, c = dof % 3;
    const int x = node % 3, y = (node / 3) % 3, zc = node / 9;
    if (x >= ix || y >= iy || zc >= iz) continue;
    float s = 0.f;
    for (int k = 0; k < kMgDenseN; ++k) s = fmaf(__ldg(M + dof * kMgDenseN + k), sb[k * kNLC + lc], s);
    z[vec_index(node_index(D, x + 1, y + 1, zc + 1), c, lc)] = s;
    if (DOT) {
      atomicAdd(&red[0][lc], (double)s * (double)s);
      atomicAdd(&red[1][lc], (double)s * (double)sb[dof * kNLC + lc]);
    }
  }
  if (DOT) {
    __syncthreads();
    if (threadIdx.x < kNLC) {
      atomicAdd(acc_zz + (int64_t)d * kNLC + threadIdx.x, red[0][threadIdx.x]);
      atomicAdd(acc_zr + (int64_t)d * kNLC + threadIdx.x, red[1][threadIdx.x]);
    }
  }
}

// -------------------------------------------------------------------------------------
// Flat CG vector kernels of the multigrid path: one thread per (active interior node, 4 load
// cases), 16-byte loads and stores, the list entry packs (domain << 40) | node.

__device__ __forceinline__ void ld4(const float* p, float (&v)[4]) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void st4(float* p, const float (&v)[4]) {
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}

// p = z + bfac p for the iterating columns (others keep p); dirf: bfac per column, NaN for a
// column that stopped
__global__ void __launch_bounds__(256) k_direction_flat(const int64_t* __restrict__ list, int64_t nitems,
                                                        const float* __restrict__ z, float* __restrict__ p,
                                                        const float* __restrict__ dirf,
                                                        const int* __restrict__ dom_active) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nitems) return;
  const int64_t e = __ldg(list + i / 6);
  const int dom = (int)(e >> kListShift);
  if (dom_active && !dom_active[dom]) return;
  const int64_t node = e & kListNodeMask;
  const int lc0 = 4 * (int)(i % 6);
  float bf[4];
  ld4(dirf + (int64_t)dom * kNLC + lc0, bf);
  bool on[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) on[j] = !isnan(bf[j]);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t k = (node * 3 + c) * kNLC + lc0;
    float zv[4], pv[4];
    ld4(z + k, zv);
    ld4(p + k, pv);
#pragma unroll
    for (int j = 0; j < 4; ++j) pv[j] = on[j] ? zv[j] + bf[j] * pv[j] : pv[j];
    st4(p + k, pv);
  }
}

// x += alpha p ; r -= alpha w (alpha per column from k_alpha, 0 for the columns that stopped),
// and t = omega D^-1 r (first step of the next V-cycle) for all four
__global__ void __launch_bounds__(256) k_update_flat(const int64_t* __restrict__ list, int64_t nitems,
                                                     float* __restrict__ x, float* __restrict__ r,
                                                     const float* __restrict__ p, const float* __restrict__ w,
                                                     const float* __restrict__ alphaf,
                                                     const float* __restrict__ binv, float omega,
                                                     float* __restrict__ t_out, const int* __restrict__ dom_active) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nitems) return;
  const int64_t e = __ldg(list + i / 6);
  const int dom = (int)(e >> kListShift);
  if (dom_active && !dom_active[dom]) return;
  const int64_t node = e & kListNodeMask;
  const int lc0 = 4 * (int)(i % 6);
  float a[4];
  ld4(alphaf + (int64_t)dom * kNLC + lc0, a);
  float rn[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const int64_t k = (node * 3 + c) * kNLC + lc0;
    float xv[4], pv[4], wv[4];
    ld4(x + k, xv);
    ld4(r + k, rn[c]);
    ld4(p + k, pv);
    ld4(w + k, wv);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      xv[j] = xv[j] + a[j] * pv[j];
      rn[c][j] = rn[c][j] - a[j] * wv[j];
    }
    st4(x + k, xv);
    st4(r + k, rn[c]);
  }
  const float2* bq = reinterpret_cast<const float2*>(binv + node * 6);   // 8-byte aligned
  const float2 q0 = __ldg(bq), q1 = __ldg(bq + 1), q2 = __ldg(bq + 2);
  const float b0 = q0.x, b1 = q0.y, b2 = q1.x, b3 = q1.y, b4 = q2.x, b5 = q2.y;
  float tv[3][4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const float r0 = rn[0][j], r1 = rn[1][j], r2 = rn[2][j];
    tv[0][j] = omega * (b0 * r0 + b3 * r1 + b4 * r2);
    tv[1][j] = omega * (b3 * r0 + b1 * r1 + b5 * r2);
    tv[2][j] = omega * (b4 * r0 + b5 * r1 + b2 * r2);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) st4(t_out + (node * 3 + c) * kNLC + lc0, tv[c]);
}

}  // namespace dtc
