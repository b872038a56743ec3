// ebe.cuh -- element-by-element stiffness application on voxel bricks (HEX08 and HEX20).
//
// One CTA owns a brick of BX x BY x BZ voxels' worth of nodes (the nodes whose fine-grid
// coordinates fall in [M*b0, M*(b0+B)) per axis, M = 1 for HEX08, 2 for HEX20) for one
// group of load cases.  It stages the nodal input of every voxel touching those nodes
// ((B+1)^3 voxels, (M*B+M+1)^3 nodes) in shared memory, lets each thread apply the element
// matrix s_v * Ke to one kept voxel for one load case, adds the rows that land on owned
// nodes into shared accumulators, and finally writes every owned node once.  Voxels on the
// brick rim are evaluated by each brick they touch (no global atomics, output written once).
// Used for HEX20 (HEX08 has the node-centric sweep of kernels.cu); the unit element matrix
// comes in as a kernel argument and is staged in shared memory.
#pragma once

namespace dtc {

// HEX20 ring-order node offsets on the doubled grid (mod_gen_quadmesh.f90:244-265)
__device__ constexpr int8_t kRingOff[20][3] = {
    {0, 0, 0}, {1, 0, 0}, {2, 0, 0}, {2, 1, 0}, {2, 2, 0}, {1, 2, 0}, {0, 2, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 1},
    {2, 2, 1}, {0, 2, 1}, {0, 0, 2}, {1, 0, 2}, {2, 0, 2}, {2, 1, 2}, {2, 2, 2}, {1, 2, 2}, {0, 2, 2}, {0, 1, 2}};

template <int NEN> struct Elem;
template <> struct Elem<8> {
  static constexpr int M = 1, ND = 24;
  static constexpr int BX = 8, BY = 8, BZ = 4;
  __host__ __device__ static constexpr int off(int a, int d) {
    return d == 0 ? ((a & 3) == 1 || (a & 3) == 2) : (d == 1 ? ((a & 3) >= 2) : (a >= 4));
  }
};
template <> struct Elem<20> {
  static constexpr int M = 2, ND = 60;
  static constexpr int BX = 4, BY = 4, BZ = 2;
  __device__ static constexpr int off(int a, int d) { return kRingOff[a][d]; }
};

template <typename T, int NEN> struct EbeShape {
  using E = Elem<NEN>;
  static constexpr int M = E::M, ND = E::ND;
  static constexpr int LCG = sizeof(T) == 4 ? 4 : 2;   // load cases per CTA
  static constexpr int NGRP = kNLC / LCG;
  static constexpr int IX = M * E::BX + M + 1, IY = M * E::BY + M + 1, IZ = M * E::BZ + M + 1;
  static constexpr int OX = M * E::BX, OY = M * E::BY, OZ = M * E::BZ;
  static constexpr int NVOX = (E::BX + 1) * (E::BY + 1) * (E::BZ + 1);
  static constexpr size_t ke_bytes = sizeof(T) * ND * ND;
  static constexpr size_t in_bytes = sizeof(T) * IX * IY * IZ * 3 * LCG;
  static constexpr size_t acc_bytes = sizeof(T) * OX * OY * OZ * 3 * LCG;
  static constexpr size_t smem = ke_bytes + in_bytes + acc_bytes + NVOX * 8 + 16 * 8;
  static constexpr int kThreadsEbe = 128;
};

// 4 consecutive floats / 2 consecutive doubles of the staged element matrix
__device__ __forceinline__ void ke_quad(const float* p, float (&v)[4]) {
  const float4 q = *reinterpret_cast<const float4*>(p);
  v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ke_quad(const double* p, double (&v)[4]) {
  const double2 a = *reinterpret_cast<const double2*>(p), b = *reinterpret_cast<const double2*>(p + 2);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// y = scale * K u on the owned nodes of one brick; ALL: every grid node, else the interior
// nodes (the unknowns); DOT: acc[col] += u . y.  ke: the unit element matrix (ND x ND,
// symmetric) in global memory; it is staged in shared memory, where every warp reads the
// same row at the same time (broadcast), so one 16-byte load feeds 4 (float) FMAs per thread.
template <typename T, int NEN, bool ALL, bool DOT>
__global__ void __launch_bounds__(128) k_ebe(const Tile* __restrict__ tiles, const DomDev* __restrict__ doms,
                                             const float* __restrict__ svox, const uint8_t* __restrict__ flags,
                                             const T* __restrict__ ke, const T* __restrict__ u, T* __restrict__ y,
                                             double scale, double* __restrict__ acc,
                                             const int* __restrict__ dom_active) {
  using S = EbeShape<T, NEN>;
  using E = Elem<NEN>;
  constexpr int M = S::M, ND = S::ND, LCG = S::LCG, NT = S::kThreadsEbe;
  static_assert(ND % 4 == 0, "element matrix rows are read 4 entries at a time");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* ske = reinterpret_cast<T*>(smem_raw);
  T* sin = reinterpret_cast<T*>(smem_raw + S::ke_bytes);
  T* sacc = reinterpret_cast<T*>(smem_raw + S::ke_bytes + S::in_bytes);
  int* vlist = reinterpret_cast<int*>(smem_raw + S::ke_bytes + S::in_bytes + S::acc_bytes);
  float* vsc = reinterpret_cast<float*>(vlist + S::NVOX);
  double* red = reinterpret_cast<double*>(vsc + S::NVOX);
  __shared__ int nv_sh;

  const Tile t = tiles[blockIdx.x / S::NGRP];
  if (dom_active && !dom_active[t.dom]) return;
  const DomDev D = doms[t.dom];
  const int g = blockIdx.x % S::NGRP;
  const int tid = threadIdx.x;
  const int ix0 = M * (t.x0 - 1), iy0 = M * (t.y0 - 1), iz0 = M * (t.z0 - 1);
  if (tid == 0) nv_sh = 0;
  if (tid < LCG) red[tid] = 0.0;
  // element matrix and input nodes: 16-byte loads, several in flight per thread
  static_assert((sizeof(T) * ND * ND) % 16 == 0, "the element matrix is copied in 16-byte pieces");
#pragma unroll 4
  for (int i = tid; i < (int)(sizeof(T) * ND * ND / 16); i += NT)
    reinterpret_cast<float4*>(ske)[i] = __ldg(reinterpret_cast<const float4*>(ke) + i);
  // stage the input nodes of the brick and its 1-voxel halo: the LCG load cases of one
  // (node, component) are 16 contiguous bytes in the vector and in the stage (one vector load)
  static_assert(sizeof(T) * LCG == 16, "one 16-byte load per (node, component)");
#pragma unroll 4
  for (int i = tid; i < S::IX * S::IY * S::IZ * 3; i += NT) {
    const int c = i % 3, nl = i / 3;
    const int gx = ix0 + nl % S::IX, gy = iy0 + (nl / S::IX) % S::IY, gz = iz0 + nl / (S::IX * S::IY);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx < D.n[0] && gy < D.n[1] && gz < D.n[2])
      v = __ldg(reinterpret_cast<const float4*>(u + vec_index(node_index(D, gx, gy, gz), c, g * LCG)));
    reinterpret_cast<float4*>(sin)[i] = v;
  }
  for (int i = tid; i < S::OX * S::OY * S::OZ * 3 * LCG; i += NT) sacc[i] = T(0);
  __syncthreads();
  // kept voxels touching the owned nodes
  for (int q = tid; q < S::NVOX; q += NT) {
    const int vx = t.x0 - 1 + q % (E::BX + 1), vy = t.y0 - 1 + (q / (E::BX + 1)) % (E::BY + 1),
              vz = t.z0 - 1 + q / ((E::BX + 1) * (E::BY + 1));
    if (vx < 0 || vy < 0 || vz < 0 || vx >= D.L[0] || vy >= D.L[1] || vz >= D.L[2]) continue;
    const float s = __ldg(svox + D.vox_off + vx + (int64_t)D.L[0] * (vy + (int64_t)D.L[1] * vz));
    if (s == 0.0f) continue;
    const int k = atomicAdd(&nv_sh, 1);
    vlist[k] = q;
    vsc[k] = s;
  }
  __syncthreads();
  const int nv = nv_sh;
  const int lo = ALL ? 0 : 1;
  const int hx = ALL ? D.n[0] - 1 : D.n[0] - 2, hy = ALL ? D.n[1] - 1 : D.n[1] - 2, hz = ALL ? D.n[2] - 1 : D.n[2] - 2;
  // work item = (kept voxel, LCT load cases, 1/SPLIT of the output nodes): every element-matrix
  // row read from shared memory feeds LCT load cases, and there are enough items for the
  // 128 threads even on bricks with few kept voxels
  constexpr int LCT = sizeof(T) == 4 ? 2 : 1, SPLIT = 4, MPER = NEN / SPLIT, NLT = LCG / LCT;
  for (int it = tid; it < nv * NLT * SPLIT; it += NT) {
    const int vi = it / (NLT * SPLIT), l0 = (it % NLT) * LCT, m0 = ((it / NLT) % SPLIT) * MPER;
    const int q = vlist[vi];
    const T s = (T)vsc[vi];
    const int qx = q % (E::BX + 1), qy = (q / (E::BX + 1)) % (E::BY + 1), qz = q / ((E::BX + 1) * (E::BY + 1));
    // local input coordinates of the voxel's origin node; fine coordinates of the voxel
    const int bx = M * qx, by = M * qy, bz = M * qz;
    const int fx = ix0 + bx, fy = iy0 + by, fz = iz0 + bz;
    T uv[ND][LCT];
#pragma unroll
    for (int a = 0; a < NEN; ++a) {
      const int nl = (bx + E::off(a, 0)) + S::IX * ((by + E::off(a, 1)) + S::IY * (bz + E::off(a, 2)));
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int j = 0; j < LCT; ++j) uv[3 * a + c][j] = sin[(nl * 3 + c) * LCG + l0 + j];
    }
#pragma unroll 1
    for (int m = m0; m < m0 + MPER; ++m) {
      const int ox = fx + E::off(m, 0), oy = fy + E::off(m, 1), oz = fz + E::off(m, 2);
      const int lx = ox - M * t.x0, ly = oy - M * t.y0, lz = oz - M * t.z0;
      const bool own = lx >= 0 && lx < S::OX && ly >= 0 && ly < S::OY && lz >= 0 && lz < S::OZ && ox >= lo &&
                       ox <= hx && oy >= lo && oy <= hy && oz >= lo && oz <= hz;
      if (!own) continue;
      T r[3][LCT];
#pragma unroll
      for (int ci = 0; ci < 3; ++ci)
#pragma unroll
        for (int j = 0; j < LCT; ++j) r[ci][j] = T(0);
      const T* krow = ske + (3 * m) * ND;
#pragma unroll
      for (int k = 0; k < ND; k += 4) {
#pragma unroll
        for (int ci = 0; ci < 3; ++ci) {
          T kv[4];
          ke_quad(krow + ci * ND + k, kv);
#pragma unroll
          for (int jj = 0; jj < 4; ++jj)
#pragma unroll
            for (int j = 0; j < LCT; ++j) r[ci][j] = fma(kv[jj], uv[k + jj][j], r[ci][j]);
        }
      }
      const int on = lx + S::OX * (ly + S::OY * lz);
#pragma unroll
      for (int ci = 0; ci < 3; ++ci)
#pragma unroll
        for (int j = 0; j < LCT; ++j) atomicAdd(&sacc[(on * 3 + ci) * LCG + l0 + j], s * r[ci][j]);
    }
  }
  __syncthreads();
  // write the owned nodes once; dot with the input at the same node
  double dot = 0.0;
  const int l = tid % LCG;   // fixed per thread: the stride is a multiple of LCG
  for (int i = tid; i < S::OX * S::OY * S::OZ * LCG; i += NT) {
    const int on = i / LCG;
    const int lx = on % S::OX, ly = (on / S::OX) % S::OY, lz = on / (S::OX * S::OY);
    const int gx = M * t.x0 + lx, gy = M * t.y0 + ly, gz = M * t.z0 + lz;
    if (gx < lo || gy < lo || gz < lo || gx > hx || gy > hy || gz > hz) continue;
    const int64_t node = node_index(D, gx, gy, gz);
    if (!(flags[node] & kNodeActive)) continue;
    const int64_t b = vec_index(node, 0, g * LCG + l);
    const int nin = (gx - ix0) + S::IX * ((gy - iy0) + S::IY * (gz - iz0));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T v = (T)(scale * D.scale * (double)sacc[(on * 3 + c) * LCG + l]);
      y[b + c * kNLC] = v;
      if (DOT) dot += (double)sin[(nin * 3 + c) * LCG + l] * (double)v;
    }
  }
  if (DOT) {
    atomicAdd(&red[l], dot);
    __syncthreads();
    if (tid < LCG) atomicAdd(acc + (int64_t)t.dom * kNLC + g * LCG + tid, red[tid]);
  }
}

}  // namespace dtc
