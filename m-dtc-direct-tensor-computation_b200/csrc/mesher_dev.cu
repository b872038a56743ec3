// mesher_dev.cu -- the reference mesh of a batch of domains on the device (sm_100a).
//
// Computes, bit for bit, what plan_mesh (mesher.cpp) computes on the host for each domain --
// gen_quadmesh_from_phi (f-src/mod_gen_quadmesh.f90:22-679) in structured form:
//   * bone voxels (phi >= llimit, :142-164, :282-316) and their element index in x-fastest
//     scan order (a per-domain prefix sum);
//   * the connected regions (:408-442): elements sharing a node are 26-neighbouring voxels,
//     so regions are 26-connected voxel components, found by a lock-free union-find
//     (hook the larger root under the smaller one with compare-and-swap, then compress), whose
//     roots are the components' first elements;
//   * the keep test (:486-553): a region is kept if one of its voxels lies on the bone bounding
//     box, the region of the first element always;
//   * the compaction quirks (:597-648): the last element and the last node always survive;
//   * node ids by first appearance over (element, local node) (:326-341): every node takes the
//     smallest key element * nen + local index over the elements that contain it; ids are the
//     ranks of the keys of the surviving nodes (a per-domain prefix sum over the keys);
//   * the constrained nodes (f-src/mod_struct_preprocess.f90:564-592): surviving nodes on the
//     domain box.
// Results go back into MeshPlan records (kept voxels, counts, quirk fields, and with
// numbering the element connectivity and the node grid indices).
//
// Work is cut into blocks of 256 items (voxels, nodes or key slots) that never cross a domain;
// a block table lists (domain, first item).  All waits are kernel boundaries; the union-find
// loop retries only when another thread changed a root, so it ends.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "mesher.h"

namespace dtc {
namespace {

constexpr int kMB = 256;   // items per block
constexpr int32_t kNoKey = 0x7f7f7f7f;   // cudaMemset pattern 0x7f: larger than every key

struct MDom {
  int32_t L[3];
  int32_t g[3];        // node grid points per edge: m*L + 1
  int32_t m, nen;
  int32_t phi_type;
  int32_t pad;
  int64_t llimit;
  int64_t vox_off;     // into the voxel arrays
  int64_t node_off;    // into the node arrays
  int64_t phi_off;     // byte offset into the gray-value upload
  int64_t slot_off;    // into the key-slot arrays (ne0 * nen per domain)
  int64_t elem_off;    // into the element arrays (ne0 per domain)
};

// per-domain results, filled by the kernels
struct MRes {
  int32_t ne0;         // bone voxels = elements before compaction
  int32_t ne_kept;     // elements of kept regions
  int32_t nn_kept;     // nodes of kept regions
  int32_t nb_kept;     // of those on the domain box
  int32_t bmin[3], bmax[3];
  int32_t last_key;    // largest first-appearance key (the last node)
  int32_t last_vox;    // voxel of the last element
};

__constant__ signed char c_mloc[20][3];   // local node offsets: HEX08 corners or HEX20 ring

__device__ __forceinline__ int64_t gray_at(const unsigned char* phi, const MDom& D, int64_t v) {
  const unsigned char* p = phi + D.phi_off;
  if (D.phi_type == 1) return (int64_t)reinterpret_cast<const int8_t*>(p)[v];
  if (D.phi_type == 2) return (int64_t)reinterpret_cast<const int16_t*>(p)[v];
  return (int64_t)reinterpret_cast<const int32_t*>(p)[v];
}

// parent[] holds domain-local voxel indices; roots satisfy parent[r] == r
// Parents always have smaller indices than their children (hooking puts the larger root under
// the smaller one, halving writes an ancestor), so every chain ends at its root.
__device__ __forceinline__ int32_t uf_find(int32_t* par, int32_t v) {
  volatile int32_t* vp = par;
  int32_t p = vp[v];
  while (p != v) {
    const int32_t gp = vp[p];
    if (gp != p) vp[v] = gp;   // path halving: a benign race, every value written is an ancestor
    v = p;
    p = gp;
  }
  return v;
}

// A failed compare-and-swap means another thread hooked the root first, i.e. progress; the
// retries are still bounded, and running out of them sets *err (the call then fails).
constexpr int kUnionRetries = 1 << 20;

__device__ void uf_union(int32_t* par, int32_t a, int32_t b, int* err) {
  for (int it = 0; it < kUnionRetries; ++it) {
    a = uf_find(par, a);
    b = uf_find(par, b);
    if (a == b) return;
    if (a < b) { const int32_t t = a; a = b; b = t; }   // hook the larger root under the smaller
    const int32_t old = atomicCAS(&par[a], a, b);
    if (old == a) return;
  }
  atomicExch(err, 1);
}

__global__ void k_bone(const int64_t* __restrict__ blk, const MDom* __restrict__ doms,
                       const unsigned char* __restrict__ phi, int32_t* __restrict__ par, uint8_t* __restrict__ bone) {
  const int64_t d = blk[2 * blockIdx.x], v = blk[2 * blockIdx.x + 1] + threadIdx.x;
  const MDom D = doms[d];
  const int64_t nv = (int64_t)D.L[0] * D.L[1] * D.L[2];
  if (v >= nv) return;
  const bool b = gray_at(phi, D, v) >= D.llimit;
  bone[D.vox_off + v] = b;
  par[D.vox_off + v] = b ? (int32_t)v : -1;
}

// one CTA per domain: element index of every bone voxel (x-fastest scan), evox, ne0, bbox
__global__ void __launch_bounds__(1024) k_elements(const MDom* __restrict__ doms, const uint8_t* __restrict__ bone,
                                                   int32_t* __restrict__ elem_of, int32_t* __restrict__ evox,
                                                   MRes* __restrict__ res) {
  __shared__ int32_t wsum[32];
  __shared__ int32_t base;
  __shared__ int32_t bb[6];
  const MDom D = doms[blockIdx.x];
  const int64_t nv = (int64_t)D.L[0] * D.L[1] * D.L[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    base = 0;
    bb[0] = bb[1] = bb[2] = INT32_MAX;
    bb[3] = bb[4] = bb[5] = -1;
  }
  __syncthreads();
  int32_t mn[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, mx[3] = {-1, -1, -1};
  for (int64_t c0 = 0; c0 < nv; c0 += 1024) {
    const int64_t v = c0 + tid;
    const int b = v < nv ? bone[D.vox_off + v] : 0;
    const unsigned bal = __ballot_sync(0xffffffffu, b);
    if (lane == 0) wsum[warp] = __popc(bal);
    __syncthreads();
    if (warp == 0) {
      const int32_t x = wsum[lane];
      int32_t s = x;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      wsum[lane] = s - x;   // exclusive prefix of the warps
    }
    __syncthreads();
    const int32_t idx = base + wsum[warp] + __popc(bal & ((1u << lane) - 1));
    if (v < nv) {
      elem_of[D.vox_off + v] = b ? idx : -1;
      if (b) {
        evox[D.elem_off + idx] = (int32_t)v;
        const int32_t x = (int32_t)(v % D.L[0]), y = (int32_t)((v / D.L[0]) % D.L[1]),
                      z = (int32_t)(v / ((int64_t)D.L[0] * D.L[1]));
        mn[0] = min(mn[0], x); mn[1] = min(mn[1], y); mn[2] = min(mn[2], z);
        mx[0] = max(mx[0], x); mx[1] = max(mx[1], y); mx[2] = max(mx[2], z);
      }
    }
    __syncthreads();
    if (tid == 1023) base = idx + b;
    __syncthreads();
  }
  for (int k = 0; k < 3; ++k) {
    atomicMin(&bb[k], mn[k]);
    atomicMax(&bb[3 + k], mx[k]);
  }
  __syncthreads();
  if (tid == 0) {
    MRes r;
    r.ne0 = base;
    r.ne_kept = r.nn_kept = r.nb_kept = 0;
    for (int k = 0; k < 3; ++k) { r.bmin[k] = bb[k]; r.bmax[k] = bb[3 + k]; }
    r.last_key = -1;
    r.last_vox = base > 0 ? evox[D.elem_off + base - 1] : -1;
    res[blockIdx.x] = r;
  }
}

// union with the 13 earlier 26-neighbours
__global__ void k_union(const int64_t* __restrict__ blk, const MDom* __restrict__ doms,
                        const uint8_t* __restrict__ bone, int32_t* __restrict__ par, int* __restrict__ err) {
  const int64_t d = blk[2 * blockIdx.x], v = blk[2 * blockIdx.x + 1] + threadIdx.x;
  const MDom D = doms[d];
  const int64_t nv = (int64_t)D.L[0] * D.L[1] * D.L[2];
  if (v >= nv || !bone[D.vox_off + v]) return;
  int32_t* p = par + D.vox_off;
  const int x = (int)(v % D.L[0]), y = (int)((v / D.L[0]) % D.L[1]), z = (int)(v / ((int64_t)D.L[0] * D.L[1]));
  for (int dz = -1; dz <= 0; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        if (dz == 0 && (dy > 0 || (dy == 0 && dx >= 0))) continue;
        const int xx = x + dx, yy = y + dy, zz = z + dz;
        if (xx < 0 || yy < 0 || zz < 0 || xx >= D.L[0] || yy >= D.L[1]) continue;
        const int64_t u = xx + (int64_t)D.L[0] * (yy + (int64_t)D.L[1] * zz);
        if (bone[D.vox_off + u]) uf_union(p, (int32_t)v, (int32_t)u, err);
      }
}

// roots; regions touching the bone bounding box (and the first element's) are kept
__global__ void k_keep(const int64_t* __restrict__ blk, const MDom* __restrict__ doms, const MRes* __restrict__ res,
                       const uint8_t* __restrict__ bone, const int32_t* __restrict__ elem_of, int32_t* __restrict__ par,
                       uint8_t* __restrict__ keepc) {
  const int64_t d = blk[2 * blockIdx.x], v = blk[2 * blockIdx.x + 1] + threadIdx.x;
  const MDom D = doms[d];
  const int64_t nv = (int64_t)D.L[0] * D.L[1] * D.L[2];
  if (v >= nv || !bone[D.vox_off + v]) return;
  int32_t* p = par + D.vox_off;
  const int32_t r = uf_find(p, (int32_t)v);
  const MRes R = res[d];
  const int x = (int)(v % D.L[0]), y = (int)((v / D.L[0]) % D.L[1]), z = (int)(v / ((int64_t)D.L[0] * D.L[1]));
  const bool touch = x == R.bmin[0] || x == R.bmax[0] || y == R.bmin[1] || y == R.bmax[1] || z == R.bmin[2] ||
                     z == R.bmax[2] || elem_of[D.vox_off + v] == 0;
  if (touch) keepc[D.vox_off + r] = 1;
}

__global__ void k_compress(const int64_t* __restrict__ blk, const MDom* __restrict__ doms,
                           const uint8_t* __restrict__ bone, int32_t* __restrict__ par) {
  const int64_t d = blk[2 * blockIdx.x], v = blk[2 * blockIdx.x + 1] + threadIdx.x;
  const MDom D = doms[d];
  const int64_t nv = (int64_t)D.L[0] * D.L[1] * D.L[2];
  if (v >= nv || !bone[D.vox_off + v]) return;
  par[D.vox_off + v] = uf_find(par + D.vox_off, (int32_t)v);
}

// kept voxels and their count; first-appearance keys of the nodes of every bone element
__global__ void k_kept_keys(const int64_t* __restrict__ blk, const MDom* __restrict__ doms,
                            const uint8_t* __restrict__ bone, const int32_t* __restrict__ elem_of,
                            const int32_t* __restrict__ par, const uint8_t* __restrict__ keepc,
                            uint8_t* __restrict__ kept, int32_t* __restrict__ key, MRes* __restrict__ res) {
  const int64_t d = blk[2 * blockIdx.x], v = blk[2 * blockIdx.x + 1] + threadIdx.x;
  const MDom D = doms[d];
  const int64_t nv = (int64_t)D.L[0] * D.L[1] * D.L[2];
  int k = 0;
  if (v < nv && bone[D.vox_off + v]) {
    k = keepc[D.vox_off + par[D.vox_off + v]];
    kept[D.vox_off + v] = (uint8_t)k;
    const int32_t e = elem_of[D.vox_off + v];
    const int x = (int)(v % D.L[0]), y = (int)((v / D.L[0]) % D.L[1]), z = (int)(v / ((int64_t)D.L[0] * D.L[1]));
    for (int a = 0; a < D.nen; ++a) {
      const int64_t g = (D.m * x + c_mloc[a][0]) + (int64_t)D.g[0] * ((D.m * y + c_mloc[a][1]) +
                                                                      (int64_t)D.g[1] * (D.m * z + c_mloc[a][2]));
      atomicMin(&key[D.node_off + g], e * D.nen + a);
    }
  } else if (v < nv) {
    kept[D.vox_off + v] = 0;
  }
  const int cnt = __syncthreads_count(k);
  if (threadIdx.x == 0 && cnt) atomicAdd(&res[d].ne_kept, cnt);
}

// nodes: survivors (component kept), the last key, counts of survivors and of those on the box
__global__ void k_nodes(const int64_t* __restrict__ blk, const MDom* __restrict__ doms,
                        const int32_t* __restrict__ key, const int32_t* __restrict__ evox,
                        const int32_t* __restrict__ par, const uint8_t* __restrict__ keepc,
                        uint8_t* __restrict__ node_keep, MRes* __restrict__ res) {
  const int64_t d = blk[2 * blockIdx.x], g = blk[2 * blockIdx.x + 1] + threadIdx.x;
  const MDom D = doms[d];
  const int64_t ng = (int64_t)D.g[0] * D.g[1] * D.g[2];
  int keep = 0, onb = 0, k = -1;
  if (g < ng) {
    k = key[D.node_off + g];
    if (k != kNoKey) {
      const int32_t v = evox[D.elem_off + k / D.nen];
      keep = keepc[D.vox_off + par[D.vox_off + v]];
      const int64_t ix = g % D.g[0], iy = (g / D.g[0]) % D.g[1], iz = g / ((int64_t)D.g[0] * D.g[1]);
      onb = ix == 0 || ix == D.g[0] - 1 || iy == 0 || iy == D.g[1] - 1 || iz == 0 || iz == D.g[2] - 1;
    } else {
      k = -1;
    }
    node_keep[D.node_off + g] = (uint8_t)keep;
  }
  const int nk = __syncthreads_count(keep), nbk = __syncthreads_count(keep && onb);
  if (threadIdx.x == 0) {
    if (nk) atomicAdd(&res[d].nn_kept, nk);
    if (nbk) atomicAdd(&res[d].nb_kept, nbk);
  }
  const int kmax = __reduce_max_sync(0xffffffffu, k);
  if ((threadIdx.x & 31) == 0 && kmax >= 0) atomicMax(&res[d].last_key, kmax);
}

// numbering: slot flag = the slot is the first appearance of a surviving node (or the last node)
__global__ void k_slot_flags(const int64_t* __restrict__ blk, const MDom* __restrict__ doms,
                             const MRes* __restrict__ res, const int32_t* __restrict__ key,
                             const int32_t* __restrict__ evox, const uint8_t* __restrict__ node_keep,
                             int32_t* __restrict__ flag, int64_t* __restrict__ slot_grid) {
  const int64_t d = blk[2 * blockIdx.x], s = blk[2 * blockIdx.x + 1] + threadIdx.x;
  const MDom D = doms[d];
  const MRes R = res[d];
  const int64_t ns = (int64_t)R.ne0 * D.nen;
  if (s >= ns) return;
  const int32_t e = (int32_t)(s / D.nen), a = (int32_t)(s % D.nen);
  const int32_t v = evox[D.elem_off + e];
  const int x = (int)(v % D.L[0]), y = (int)((v / D.L[0]) % D.L[1]), z = (int)(v / ((int64_t)D.L[0] * D.L[1]));
  const int64_t g = (D.m * x + c_mloc[a][0]) + (int64_t)D.g[0] * ((D.m * y + c_mloc[a][1]) +
                                                                  (int64_t)D.g[1] * (D.m * z + c_mloc[a][2]));
  slot_grid[D.slot_off + s] = g;
  const bool first = key[D.node_off + g] == (int32_t)s;
  flag[D.slot_off + s] = first && (node_keep[D.node_off + g] || (int32_t)s == R.last_key);
}

// per-block sums of a flag array over the block table, then per-domain exclusive scans
__global__ void k_block_sums(const int64_t* __restrict__ blk, int64_t nblk, const int64_t* __restrict__ item_off,
                             const int64_t* __restrict__ item_n, const int32_t* __restrict__ flag,
                             int32_t* __restrict__ bsum) {
  const int64_t b = blockIdx.x;
  const int64_t d = blk[2 * b], i = blk[2 * b + 1] + threadIdx.x;
  const int f = i < item_n[d] ? flag[item_off[d] + i] : 0;
  const int c = __syncthreads_count(f);
  if (threadIdx.x == 0) bsum[b] = c;
}

// exclusive scan of the block sums of each domain (one CTA per domain, blocks of a domain are
// consecutive in the table), then of the items inside each block
__global__ void k_scan_blocks(const int64_t* __restrict__ dom_blk0, const int64_t* __restrict__ dom_nblk,
                              int32_t* __restrict__ bsum) {
  const int64_t b0 = dom_blk0[blockIdx.x], nb = dom_nblk[blockIdx.x];
  if (threadIdx.x != 0) return;
  int32_t run = 0;
  for (int64_t b = 0; b < nb; ++b) {
    const int32_t c = bsum[b0 + b];
    bsum[b0 + b] = run;
    run += c;
  }
}

__global__ void k_scan_items(const int64_t* __restrict__ blk, const int64_t* __restrict__ item_off,
                             const int64_t* __restrict__ item_n, const int32_t* __restrict__ flag,
                             const int32_t* __restrict__ bsum, int32_t* __restrict__ rank) {
  __shared__ int32_t wsum[8];
  const int64_t b = blockIdx.x;
  const int64_t d = blk[2 * b], i = blk[2 * b + 1] + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int f = i < item_n[d] ? flag[item_off[d] + i] : 0;
  const unsigned bal = __ballot_sync(0xffffffffu, f);
  if (lane == 0) wsum[warp] = __popc(bal);
  __syncthreads();
  int32_t off = bsum[b];
  for (int w = 0; w < warp; ++w) off += wsum[w];
  if (i < item_n[d]) rank[item_off[d] + i] = off + __popc(bal & ((1u << lane) - 1));
}

// output elements: those of kept regions and the last one
__global__ void k_elem_flags(const int64_t* __restrict__ blk, const MDom* __restrict__ doms,
                             const MRes* __restrict__ res, const int32_t* __restrict__ evox,
                             const uint8_t* __restrict__ kept, int32_t* __restrict__ eflag) {
  const int64_t d = blk[2 * blockIdx.x], e = blk[2 * blockIdx.x + 1] + threadIdx.x;
  const MDom D = doms[d];
  const MRes R = res[d];
  if (e >= R.ne0) return;
  eflag[D.elem_off + e] = kept[D.vox_off + evox[D.elem_off + e]] || e == R.ne0 - 1;
}

// element list in reference order: kept elements and the last one; node id of a slot
__global__ void k_emit_elems(const int64_t* __restrict__ blk, const MDom* __restrict__ doms,
                             const MRes* __restrict__ res, const int32_t* __restrict__ evox,
                             const uint8_t* __restrict__ kept, const int32_t* __restrict__ erank,
                             const int32_t* __restrict__ key, const int32_t* __restrict__ srank,
                             const int32_t* __restrict__ sflag, const int64_t* __restrict__ slot_grid,
                             int64_t* __restrict__ elems) {
  const int64_t d = blk[2 * blockIdx.x], s = blk[2 * blockIdx.x + 1] + threadIdx.x;
  const MDom D = doms[d];
  const MRes R = res[d];
  const int64_t ns = (int64_t)R.ne0 * D.nen;
  if (s >= ns) return;
  const int32_t e = (int32_t)(s / D.nen), a = (int32_t)(s % D.nen);
  const int32_t v = evox[D.elem_off + e];
  const bool out = kept[D.vox_off + v] || e == R.ne0 - 1;
  if (!out) return;
  const int64_t g = slot_grid[D.slot_off + s];
  const int32_t k = key[D.node_off + g];
  const int64_t id = sflag[D.slot_off + k] ? (int64_t)srank[D.slot_off + k] + 1 : 0;
  elems[D.slot_off + (int64_t)erank[D.elem_off + e] * D.nen + a] = id;
}

}  // namespace

// Meshes n domains on the current device; plans[i] receives exactly what plan_mesh gives.
int mesh_batch_device(const dtc_domain_in* in, int64_t n, MeshPlan* plans, bool numbering, void* stream,
                      std::string& msg) {
  if (n <= 0) return DTC_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  static const signed char kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
                                            {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
  static const signed char kRing[20][3] = {{0, 0, 0}, {1, 0, 0}, {2, 0, 0}, {2, 1, 0}, {2, 2, 0}, {1, 2, 0},
                                           {0, 2, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 1}, {2, 2, 1}, {0, 2, 1},
                                           {0, 0, 2}, {1, 0, 2}, {2, 0, 2}, {2, 1, 2}, {2, 2, 2}, {1, 2, 2},
                                           {0, 2, 2}, {0, 1, 2}};
  const int nen = in[0].elem_type;
  for (int64_t i = 0; i < n; ++i) {
    if (in[i].elem_type != nen) { msg = "device mesher: one element type per batch"; return DTC_ERR_INVALID_ARGUMENT; }
    for (int d = 0; d < 3; ++d)
      if (in[i].L[d] < 1 || in[i].L[d] > 4096) { msg = "device mesher: L out of range"; return DTC_ERR_INVALID_ARGUMENT; }
  }
  for (int64_t i = 0; i < n; ++i)
    if (in[i].L[0] * in[i].L[1] * in[i].L[2] * (int64_t)nen >= (int64_t)kNoKey) {
      msg = "device mesher: domain too large for 32-bit first-appearance keys";
      return DTC_ERR_INVALID_ARGUMENT;
    }
  signed char loc[20][3];
  std::memset(loc, 0, sizeof(loc));
  std::memcpy(loc, nen == 8 ? &kCorner[0][0] : &kRing[0][0], (size_t)nen * 3);
  DTC_CUDA(cudaMemcpyToSymbolAsync(c_mloc, loc, sizeof(loc), 0, cudaMemcpyHostToDevice, s));
  const int m = nen == 8 ? 1 : 2;
  std::vector<MDom> doms((size_t)n);
  int64_t vox = 0, nodes = 0, phib = 0;
  for (int64_t i = 0; i < n; ++i) {
    MDom& D = doms[i];
    std::memset(&D, 0, sizeof(D));
    for (int d = 0; d < 3; ++d) { D.L[d] = (int32_t)in[i].L[d]; D.g[d] = m * D.L[d] + 1; }
    D.m = m; D.nen = nen; D.phi_type = in[i].phi_type; D.llimit = in[i].llimit;
    D.vox_off = vox; D.node_off = nodes; D.phi_off = phib;
    const int64_t nv = (int64_t)D.L[0] * D.L[1] * D.L[2];
    vox += nv;
    nodes += (int64_t)D.g[0] * D.g[1] * D.g[2];
    phib += ((nv * in[i].phi_type + 15) / 16) * 16;
  }
  // block tables over voxels and nodes
  std::vector<int64_t> vblk, nblk;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t nv = (int64_t)doms[i].L[0] * doms[i].L[1] * doms[i].L[2];
    const int64_t ng = (int64_t)doms[i].g[0] * doms[i].g[1] * doms[i].g[2];
    for (int64_t q = 0; q < nv; q += kMB) { vblk.push_back(i); vblk.push_back(q); }
    for (int64_t q = 0; q < ng; q += kMB) { nblk.push_back(i); nblk.push_back(q); }
  }
  // device scratch (stream-ordered allocations: no device-wide synchronisation)
  std::vector<void*> owned;
  auto alloc = [&](size_t bytes, void** p) -> cudaError_t {
    cudaError_t e = cudaMallocAsync(p, std::max<size_t>(bytes, 16), s);
    if (e == cudaSuccess) owned.push_back(*p);
    return e;
  };
  auto release = [&]() {
    for (void* p : owned) cudaFreeAsync(p, s);
    owned.clear();
  };
  unsigned char* dphi = nullptr;
  MDom* ddoms = nullptr;
  MRes* dres = nullptr;
  int64_t *dvblk = nullptr, *dnblk = nullptr;
  int32_t *par = nullptr, *elem_of = nullptr, *evox = nullptr, *key = nullptr;
  uint8_t *bone = nullptr, *keepc = nullptr, *kept = nullptr, *node_keep = nullptr;
  int* derr = nullptr;
  cudaError_t e;
  auto fail = [&](cudaError_t err, const char* what) {
    msg = std::string("device mesher: ") + what + ": " + cudaGetErrorString(err);
    release();
    return err == cudaErrorMemoryAllocation ? DTC_ERR_OUT_OF_MEMORY : DTC_ERR_CUDA;
  };
  if ((e = alloc(phib, (void**)&dphi)) || (e = alloc(sizeof(MDom) * n, (void**)&ddoms)) ||
      (e = alloc(sizeof(MRes) * n, (void**)&dres)) || (e = alloc(sizeof(int64_t) * vblk.size(), (void**)&dvblk)) ||
      (e = alloc(sizeof(int64_t) * nblk.size(), (void**)&dnblk)) || (e = alloc(sizeof(int32_t) * vox, (void**)&par)) ||
      (e = alloc(sizeof(int32_t) * vox, (void**)&elem_of)) || (e = alloc(sizeof(int32_t) * vox, (void**)&evox)) ||
      (e = alloc(sizeof(int32_t) * nodes, (void**)&key)) || (e = alloc(vox, (void**)&bone)) ||
      (e = alloc(vox, (void**)&keepc)) || (e = alloc(vox, (void**)&kept)) || (e = alloc(nodes, (void**)&node_keep)) ||
      (e = alloc(sizeof(int), (void**)&derr)))
    return fail(e, "allocation");
  // element offsets: a voxel bound (ne0 <= voxels) so that no count is needed up front
  for (int64_t i = 0; i < n; ++i) doms[i].elem_off = doms[i].vox_off;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t nv = (int64_t)doms[i].L[0] * doms[i].L[1] * doms[i].L[2];
    if ((e = cudaMemcpyAsync(dphi + doms[i].phi_off, in[i].phi, (size_t)(nv * in[i].phi_type), cudaMemcpyHostToDevice,
                             s)))
      return fail(e, "gray values");
  }
  if ((e = cudaMemcpyAsync(dvblk, vblk.data(), sizeof(int64_t) * vblk.size(), cudaMemcpyHostToDevice, s)) ||
      (e = cudaMemcpyAsync(dnblk, nblk.data(), sizeof(int64_t) * nblk.size(), cudaMemcpyHostToDevice, s)) ||
      (e = cudaMemsetAsync(keepc, 0, vox, s)) || (e = cudaMemsetAsync(key, 0x7f, sizeof(int32_t) * nodes, s)) ||
      (e = cudaMemsetAsync(derr, 0, sizeof(int), s)))
    return fail(e, "set-up");
  // (the slot offsets of the numbering follow once ne0 is known; the first kernels do not read them)
  if ((e = cudaMemcpyAsync(ddoms, doms.data(), sizeof(MDom) * n, cudaMemcpyHostToDevice, s))) return fail(e, "domains");
  const unsigned nvb = (unsigned)(vblk.size() / 2), nnb = (unsigned)(nblk.size() / 2);
  k_bone<<<nvb, kMB, 0, s>>>(dvblk, ddoms, dphi, par, bone);
  k_elements<<<(unsigned)n, 1024, 0, s>>>(ddoms, bone, elem_of, evox, dres);
  k_union<<<nvb, kMB, 0, s>>>(dvblk, ddoms, bone, par, derr);
  k_keep<<<nvb, kMB, 0, s>>>(dvblk, ddoms, dres, bone, elem_of, par, keepc);
  k_compress<<<nvb, kMB, 0, s>>>(dvblk, ddoms, bone, par);
  if ((e = cudaGetLastError())) return fail(e, "components");
  k_kept_keys<<<nvb, kMB, 0, s>>>(dvblk, ddoms, bone, elem_of, par, keepc, kept, key, dres);
  k_nodes<<<nnb, kMB, 0, s>>>(dnblk, ddoms, key, evox, par, keepc, node_keep, dres);
  if ((e = cudaGetLastError())) return fail(e, "nodes");
  std::vector<MRes> hres((size_t)n);
  std::vector<uint8_t> hkept((size_t)vox);
  int herr = 0;
  if ((e = cudaMemcpyAsync(hres.data(), dres, sizeof(MRes) * n, cudaMemcpyDeviceToHost, s)) ||
      (e = cudaMemcpyAsync(hkept.data(), kept, vox, cudaMemcpyDeviceToHost, s)) ||
      (e = cudaMemcpyAsync(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost, s)) || (e = cudaStreamSynchronize(s)))
    return fail(e, "results");
  if (herr) { msg = "device mesher: union-find retries ran out"; release(); return DTC_ERR_INTERNAL; }
  // per-domain records, as plan_mesh writes them
  for (int64_t i = 0; i < n; ++i) {
    MeshPlan& mp = plans[i];
    mp = MeshPlan();
    mp.nen = nen;
    for (int d = 0; d < 3; ++d) mp.L[d] = in[i].L[d];
    const MRes& R = hres[i];
    const MDom& D = doms[i];
    if (R.ne0 == 0) { mp.status = DTC_DOMAIN_EMPTY; continue; }
    const int64_t nv = (int64_t)D.L[0] * D.L[1] * D.L[2];
    mp.kept.assign(hkept.begin() + D.vox_off, hkept.begin() + D.vox_off + nv);
    const int64_t vlast = R.last_vox;   // the last element's voxel: the last bone voxel in scan order
    mp.last_voxel = vlast;
    const bool last_kept = mp.kept[vlast] != 0;
    int64_t ne = R.ne_kept, nn = R.nn_kept, nb = R.nb_kept;
    if (!last_kept) { mp.last_partial = true; ++ne; }
    // the last node: its key is the largest; it survives even outside the kept regions
    const int32_t lk = R.last_key;
    const int32_t a = lk % nen;
    const int64_t vx = vlast % D.L[0], vy = (vlast / D.L[0]) % D.L[1], vz = vlast / ((int64_t)D.L[0] * D.L[1]);
    const int64_t g = (m * vx + loc[a][0]) + (int64_t)D.g[0] * ((m * vy + loc[a][1]) + (int64_t)D.g[1] * (m * vz + loc[a][2]));
    const int64_t ix = g % D.g[0], iy = (g / D.g[0]) % D.g[1], iz = g / ((int64_t)D.g[0] * D.g[1]);
    const bool lonb = ix == 0 || ix == D.g[0] - 1 || iy == 0 || iy == D.g[1] - 1 || iz == 0 || iz == D.g[2] - 1;
    if (!last_kept) {
      // the last node lies in the last element; its region was dropped, so it is counted here
      ++nn;
      nb += lonb;
      mp.last_grid = g;
      mp.last_on_boundary = lonb;
      mp.last_local = a;
    }
    mp.ne = ne; mp.nn = nn; mp.nb = nb;
    mp.n_free_dof = 3 * (nn - nb);
    if (nn == 0 || ne == 0) { mp.status = DTC_DOMAIN_NO_STRUCTURE; continue; }
    if (nn < 6) mp.status = DTC_DOMAIN_FEW_NODES;
  }
  if (numbering) {
    // slots (element, local node) of each domain; element and slot ranks by per-domain scans
    std::vector<int64_t> sblk, eblk, s_off(n), s_n(n), e_off(n), e_n(n), sdom0(n), sdomn(n), edom0(n), edomn(n);
    int64_t slots = 0;
    for (int64_t i = 0; i < n; ++i) {
      doms[i].slot_off = slots;
      s_off[i] = slots; s_n[i] = (int64_t)hres[i].ne0 * nen;
      e_off[i] = doms[i].elem_off; e_n[i] = hres[i].ne0;
      slots += s_n[i];
      sdom0[i] = (int64_t)sblk.size() / 2;
      for (int64_t q = 0; q < s_n[i]; q += kMB) { sblk.push_back(i); sblk.push_back(q); }
      sdomn[i] = (int64_t)sblk.size() / 2 - sdom0[i];
      edom0[i] = (int64_t)eblk.size() / 2;
      for (int64_t q = 0; q < e_n[i]; q += kMB) { eblk.push_back(i); eblk.push_back(q); }
      edomn[i] = (int64_t)eblk.size() / 2 - edom0[i];
    }
    int32_t *sflag = nullptr, *srank = nullptr, *eflag = nullptr, *erank = nullptr, *sbs = nullptr, *ebs = nullptr;
    int64_t *sgrid = nullptr, *elems = nullptr, *dsblk = nullptr, *deblk = nullptr, *meta = nullptr;
    const size_t nsb = sblk.size() / 2, neb = eblk.size() / 2;
    if ((e = alloc(sizeof(int32_t) * slots, (void**)&sflag)) || (e = alloc(sizeof(int32_t) * slots, (void**)&srank)) ||
        (e = alloc(sizeof(int32_t) * vox, (void**)&eflag)) || (e = alloc(sizeof(int32_t) * vox, (void**)&erank)) ||
        (e = alloc(sizeof(int32_t) * std::max<size_t>(nsb, 1), (void**)&sbs)) ||
        (e = alloc(sizeof(int32_t) * std::max<size_t>(neb, 1), (void**)&ebs)) ||
        (e = alloc(sizeof(int64_t) * slots, (void**)&sgrid)) || (e = alloc(sizeof(int64_t) * slots, (void**)&elems)) ||
        (e = alloc(sizeof(int64_t) * sblk.size(), (void**)&dsblk)) ||
        (e = alloc(sizeof(int64_t) * eblk.size(), (void**)&deblk)) || (e = alloc(sizeof(int64_t) * 8 * n, (void**)&meta)))
      return fail(e, "allocation");
    std::vector<int64_t> hmeta(8 * n);
    for (int64_t i = 0; i < n; ++i) {
      hmeta[i] = s_off[i]; hmeta[n + i] = s_n[i]; hmeta[2 * n + i] = e_off[i]; hmeta[3 * n + i] = e_n[i];
      hmeta[4 * n + i] = sdom0[i]; hmeta[5 * n + i] = sdomn[i]; hmeta[6 * n + i] = edom0[i]; hmeta[7 * n + i] = edomn[i];
    }
    if ((e = cudaMemcpyAsync(ddoms, doms.data(), sizeof(MDom) * n, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(dsblk, sblk.data(), sizeof(int64_t) * sblk.size(), cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(deblk, eblk.data(), sizeof(int64_t) * eblk.size(), cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(meta, hmeta.data(), sizeof(int64_t) * hmeta.size(), cudaMemcpyHostToDevice, s)))
      return fail(e, "numbering set-up");
    if (neb) k_elem_flags<<<(unsigned)neb, kMB, 0, s>>>(deblk, ddoms, dres, evox, kept, eflag);
    if (nsb) {
      k_slot_flags<<<(unsigned)nsb, kMB, 0, s>>>(dsblk, ddoms, dres, key, evox, node_keep, sflag, sgrid);
      k_block_sums<<<(unsigned)nsb, kMB, 0, s>>>(dsblk, (int64_t)nsb, meta, meta + n, sflag, sbs);
      k_scan_blocks<<<(unsigned)n, 32, 0, s>>>(meta + 4 * n, meta + 5 * n, sbs);
      k_scan_items<<<(unsigned)nsb, kMB, 0, s>>>(dsblk, meta, meta + n, sflag, sbs, srank);
    }
    if (neb) {
      k_block_sums<<<(unsigned)neb, kMB, 0, s>>>(deblk, (int64_t)neb, meta + 2 * n, meta + 3 * n, eflag, ebs);
      k_scan_blocks<<<(unsigned)n, 32, 0, s>>>(meta + 6 * n, meta + 7 * n, ebs);
      k_scan_items<<<(unsigned)neb, kMB, 0, s>>>(deblk, meta + 2 * n, meta + 3 * n, eflag, ebs, erank);
    }
    if (nsb)
      k_emit_elems<<<(unsigned)nsb, kMB, 0, s>>>(dsblk, ddoms, dres, evox, kept, erank, key, srank, sflag, sgrid,
                                                 elems);
    if ((e = cudaGetLastError())) return fail(e, "numbering");
    std::vector<int64_t> helems((size_t)slots), hgrid((size_t)slots);
    std::vector<int32_t> hsflag((size_t)slots), hsrank((size_t)slots);
    if ((e = cudaMemcpyAsync(helems.data(), elems, sizeof(int64_t) * slots, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(hgrid.data(), sgrid, sizeof(int64_t) * slots, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(hsflag.data(), sflag, sizeof(int32_t) * slots, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(hsrank.data(), srank, sizeof(int32_t) * slots, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaStreamSynchronize(s)))
      return fail(e, "numbering results");
    for (int64_t i = 0; i < n; ++i) {
      MeshPlan& mp = plans[i];
      if (mp.status == DTC_DOMAIN_EMPTY) continue;
      mp.elems.assign(helems.begin() + s_off[i], helems.begin() + s_off[i] + mp.ne * nen);
      mp.node_grid.assign((size_t)mp.nn, 0);
      for (int64_t q = 0; q < s_n[i]; ++q)
        if (hsflag[s_off[i] + q]) {
          const int64_t r = hsrank[s_off[i] + q];
          if (r < 0 || r >= mp.nn) { msg = "device mesher: inconsistent node ranks"; release(); return DTC_ERR_INTERNAL; }
          mp.node_grid[r] = hgrid[s_off[i] + q];
        }
    }
  }
  release();
  if ((e = cudaStreamSynchronize(s))) return fail(e, "release");
  return DTC_OK;
}

}  // namespace dtc
