// matvec_tc.cu -- the voxel stiffness contraction on the 5th-generation tensor cores (sm_100a).
//
// HEX08 (k_sweep_tc): the three fine-level sweeps of the FP32 inner solve -- the CG operator
// application, the multigrid residual and the post-smoothing -- with the 24 x 24 voxel
// contraction as tcgen05.mma kind::tf32, A (voxel DOFs x load cases) in tensor memory, B (the
// unit voxel stiffness) in shared memory.  HEX20 (k_ebe_tc): the 60 x 60 element contraction
// of the brick kernel, A and B in shared memory.  Both split FP32 operands into tf32 hi + lo
// parts (three products) for FP32-level accuracy and bound every wait.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/dtc.h"
#include "kernels.cuh"

namespace dtc {

namespace tc {

constexpr int kRows = 128;                 // M: 16 voxels x 8 load cases
constexpr int kVoxPerRound = 16;
constexpr int kK = 24, kN = 32, kKc = 8;   // voxel DOFs, padded output DOFs, K per MMA
constexpr int kMaxVox = 9 * 5 * 5;         // voxels adjacent to an 8 x 4 x 4 node tile
constexpr int kAChunkBytes = kRows * kKc * 4;   // 4 KB: one K-chunk of A in canonical layout
constexpr int kBChunkBytes = kN * kKc * 4;      // 1 KB
constexpr uint32_t kTmemCols = 32;
constexpr long long kSpinLimit = 1ll << 26;

// Canonical K-major, no-swizzle layout of a (rows x 8) tf32 chunk: 8-row x 16-byte core
// matrices; the two K-halves of a row group are LBO = 128 B apart, row groups SBO = 256 B.
__host__ __device__ constexpr int canon_offset(int r, int k) {
  return (r & 7) * 16 + (r >> 3) * 256 + ((k >> 2) & 1) * 128 + (k & 3) * 4;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
  d |= (uint64_t)((128 >> 4) & 0x3FFF) << 16;      // leading byte offset (K direction)
  d |= (uint64_t)((256 >> 4) & 0x3FFF) << 32;      // stride byte offset (M/N direction)
  d |= (uint64_t)1 << 46;                           // descriptor version (sm100)
  // base offset 0, lbo mode 0, layout type 0 = SWIZZLE_NONE
  return d;
}

// instruction descriptor: D f32, A/B tf32, both K-major, N = 32, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kN >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// Waits until the mbarrier phase of the given parity has completed: one immediate test, then
// up to limit - 1 potentially suspending polls.  Returns false when the limit runs out (at
// once for limit <= 0).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit = kSpinLimit) {
  if (limit <= 0) return false;
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  if (done) return true;
  for (long long i = 1; i < limit; ++i) {
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace tc

// Polls of the per-round completion wait before a kernel gives up (the drain wait before the
// tensor memory is freed always keeps the full bound).  dtc_options.tc_wait_spins sets it.
__device__ long long g_tc_spin_limit = tc::kSpinLimit;

int set_tc_spin_limit(long long spins, cudaStream_t s, std::string& msg) {
  const long long v = spins > 0 ? spins : spins == 0 ? tc::kSpinLimit : 0;
  DTC_CUDA(cudaMemcpyToSymbolAsync(g_tc_spin_limit, &v, sizeof(v), 0, cudaMemcpyHostToDevice, s));
  DTC_CUDA(cudaStreamSynchronize(s));   // v lives on this stack frame
  return DTC_OK;
}

// -------------------------------------------------------------------------------------
// HEX08 sweeps of the FP32 inner solve on the tensor cores.
//
// One CTA = one node tile (8 x 4 x 4 owned nodes) x one group of 8 load cases; it evaluates
// every kept voxel adjacent to an owned node.  A round takes 16 of these voxels: thread
// tid owns row tid of the MMA (voxel tid / 8 of the round, load case tid % 8), loads that
// voxel's 24 corner DOFs of its load case straight from the nodal vector into registers,
// splits them into tf32 hi + lo and stores the two halves into its own tensor-memory lane
// (the A operand, columns 0-23 and 24-47).  One thread then issues
//     D = A_hi B_hi + A_hi B_lo + A_lo B_hi      (B = Khat, split on the host; 3 K-chunks)
// as nine tcgen05.mma kind::tf32 (M = 128, N = 32, K = 8) with A read from tensor memory and
// B from shared memory, into one of two 32-column accumulators.  While those run, every
// thread reads the previous round's accumulator row (tcgen05.ld: the voxel's 24 outputs),
// scales it by the voxel's modulus factor and adds the outputs of owned nodes into shared
// memory.  After the last round the owned active nodes get the sweep's own epilogue:
//   kTcApply: y = scale * K u,                              acc1 += u . y  (CG: p . K p)
//   kTcRes  : y = b - K u                                   (multigrid residual)
//   kTcPost : y = u + omega D^-1 (b - K u),  acc1 += y . y, acc2 += y . b   (post-smoothing)
// Precision: the split recovers FP32-level products (the tf32 rounding of the lo parts costs
// at most 2^-21 relative); accumulation is FP32 in tensor memory, then FP64 for the scale.
// Waits: every completion wait is bounded by g_tc_spin_limit polls; on time-out the CTA
// records the error, waits (full bound) for the MMAs it committed, frees its tensor memory
// and returns.
namespace tc {
constexpr int kSweepVox = 16;                        // voxels per round (x 8 load cases = 128 rows)
constexpr uint32_t kColAHi = 0, kColALo = 24;        // A operand columns
constexpr uint32_t kColD0 = 64, kColD1 = 96;         // the two accumulators
constexpr uint32_t kSweepCols = 128;                 // tensor-memory columns per CTA
constexpr int kSweepAccBytes = 128 * 3 * 8 * 4;      // owned node x comp x load case (floats)
// dynamic shared memory per CTA: B (6 KB) + accumulators (12 KB), padded so that at most four
// CTAs share an SM (4 x 128 columns = the SM's 512 tensor-memory columns)
constexpr int kSweepSmem = 52 * 1024;

__device__ __forceinline__ void mma_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t accumulate) {
  uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "r"(tmem_a), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// local corner lm (the mesher's HEX08 order) -> offsets
__device__ __forceinline__ int corner_dx(int lm) { return (lm == 1 || lm == 2 || lm == 5 || lm == 6) ? 1 : 0; }
__device__ __forceinline__ int corner_dy(int lm) { return (lm == 2 || lm == 3 || lm == 6 || lm == 7) ? 1 : 0; }
__device__ __forceinline__ int corner_dz(int lm) { return lm >= 4 ? 1 : 0; }
}  // namespace tc

// Khat split into tf32 hi / lo, laid out as 6 canonical B chunks (hi k0..2, lo k0..2).
__constant__ float c_bsplit[6 * tc::kN * tc::kKc];

template <int MODE>
__global__ void __launch_bounds__(128, 4)
    k_sweep_tc(const Tile* __restrict__ tiles, const DomDev* __restrict__ doms, const float* __restrict__ svox,
               const uint8_t* __restrict__ flags, const float* __restrict__ binv, const float* __restrict__ b,
               const float* __restrict__ u, float* __restrict__ y, float scale, float omega,
               double* __restrict__ acc1, double* __restrict__ acc2, const int* __restrict__ dom_active,
               int* __restrict__ err) {
  using namespace tc;
  extern __shared__ __align__(1024) unsigned char dsm[];
  unsigned char* sB = dsm;                                        // 6 KB, canonical K-major chunks
  float* acc = reinterpret_cast<float*>(dsm + 6 * kBChunkBytes);   // 12 KB
  __shared__ int vlist[kMaxVox];
  __shared__ float vscale[kMaxVox];
  __shared__ int vown[kMaxVox];   // owned corners (8 bits) | (local node of corner 0 + 64) << 8
  __shared__ int wcount[4];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ int fail;
  __shared__ double red[32];

  const Tile t = tiles[blockIdx.x / 3];
  if (dom_active && !dom_active[t.dom]) return;
  const DomDev D = doms[t.dom];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = blockIdx.x % 3;  // load-case group: the three groups of a tile run back to back

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(kSweepCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  for (int i = tid; i < 6 * kN * kKc; i += 128) reinterpret_cast<float*>(sB)[i] = c_bsplit[i];
  for (int i = tid; i < 128 * 3 * 8; i += 128) acc[i] = 0.0f;

  // kept voxels adjacent to the owned nodes, in x-fastest order
  const int L0 = D.L[0], L1 = D.L[1], L2 = D.L[2];
  int nv = 0;
  for (int base = 0; base < kMaxVox; base += 128) {
    const int q = base + tid;
    int vidx = -1;
    float sv = 0.0f;
    if (q < kMaxVox) {
      const int ix = q % 9, iy = (q / 9) % 5, iz = q / 45;
      const int vx = t.x0 - 1 + ix, vy = t.y0 - 1 + iy, vz = t.z0 - 1 + iz;
      if (vx >= 0 && vy >= 0 && vz >= 0 && vx < L0 && vy < L1 && vz < L2) {
        sv = __ldg(svox + D.vox_off + vx + (int64_t)L0 * (vy + (int64_t)L1 * vz));
        if (sv != 0.0f) vidx = vx | (vy << 10) | (vz << 20);   // packed: no divisions in the rounds
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, vidx >= 0);
    if (lane == 0) wcount[warp] = __popc(m);
    __syncthreads();
    int off = nv;
    for (int w2 = 0; w2 < warp; ++w2) off += wcount[w2];
    if (vidx >= 0) {
      const int pos = off + __popc(m & ((1u << lane) - 1));
      vlist[pos] = vidx;
      vscale[pos] = sv;
      const int vx = vidx & 1023, vy = (vidx >> 10) & 1023, vz = vidx >> 20;
      int own = 0;
#pragma unroll
      for (int lm = 0; lm < 8; ++lm) {
        const int ox = vx + corner_dx(lm), oy = vy + corner_dy(lm), oz = vz + corner_dz(lm);
        const int lx = ox - t.x0, ly = oy - t.y0, lz = oz - t.z0;
        if (lx >= 0 && lx < kTileX && ly >= 0 && ly < kTileY && lz >= 0 && lz < kTileZ && ox >= 1 &&
            ox <= D.n[0] - 2 && oy >= 1 && oy <= D.n[1] - 2 && oz >= 1 && oz <= D.n[2] - 2)
          own |= 1 << lm;
      }
      vown[pos] = own | ((vx - t.x0 + kTileX * ((vy - t.y0) + kTileY * (vz - t.z0)) + 64) << 8);
    }
    nv += wcount[0] + wcount[1] + wcount[2] + wcount[3];
    __syncthreads();
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // B visible to the tensor cores
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t sB_addr = smem_u32(sB);
  const int lcl = tid & 7, lc = g * kLcGroup + lcl;
  const int rounds = (nv + kSweepVox - 1) / kSweepVox;
  const long long lim = g_tc_spin_limit;
  const int64_t nx = D.n[0], nxy = (int64_t)D.n[0] * D.n[1];
  const int hi_x = D.n[0] - 2, hi_y = D.n[1] - 2, hi_z = D.n[2] - 2;

  // the voxel's 24 corner DOFs of this thread's load case for round rd (zero rows past the list)
  auto gather = [&](int rd, float (&a)[24]) {
    const int vs = rd * kSweepVox + (tid >> 3);
    if (vs < nv) {
      const int vi = vlist[vs];
      const int vx = vi & 1023, vy = (vi >> 10) & 1023, vz = vi >> 20;
      const int64_t n0 = D.node_off + vx + nx * vy + nxy * vz;
#pragma unroll
      for (int lm = 0; lm < 8; ++lm) {
        const int64_t nb = vec_index(n0 + corner_dx(lm) + nx * corner_dy(lm) + nxy * corner_dz(lm), 0, lc);
#pragma unroll
        for (int c = 0; c < 3; ++c) a[3 * lm + c] = __ldg(u + nb + c * kNLC);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 24; ++k) a[k] = 0.0f;
    }
  };
  float a[24];
  if (rounds > 0) gather(0, a);
  int committed = 0;
  for (int rd = 0; rd <= rounds; ++rd) {
    // (1) this round's A row, split into tf32 hi + lo (its loads were issued an iteration ago)
    uint32_t av[48];
    if (rd < rounds) {
#pragma unroll
      for (int k = 0; k < 24; ++k) {
        const uint32_t hb = __float_as_uint(a[k]) & 0xFFFFE000u;   // tf32 hi: exact, low 13 bits clear
        av[k] = hb;
        av[24 + k] = __float_as_uint(a[k] - __uint_as_float(hb));
      }
    }
    // (2) the MMAs of the previous round have finished: A is free, its accumulator is ready
    if (rd >= 1 && !mbar_wait(smem_u32(&mbar), (uint32_t)((rd - 1) & 1), lim)) atomicOr(&fail, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // (3) store A, then one thread issues this round's MMAs
    if (rd < rounds) {
      tmem_st16(lane_addr + kColAHi, av);
      tmem_st16(lane_addr + kColAHi + 16, av + 16);
      tmem_st16(lane_addr + kColAHi + 32, av + 32);
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (fail) break;
    if (rd < rounds) {
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + ((rd & 1) ? kColD1 : kColD0);
#pragma unroll
        for (int kc = 0; kc < 3; ++kc) {
          const uint64_t bhi = smem_desc(sB_addr + kc * kBChunkBytes), blo = smem_desc(sB_addr + (3 + kc) * kBChunkBytes);
          mma_ts(d, tmem + kColAHi + 8 * kc, bhi, kc > 0 ? 1u : 0u);
          mma_ts(d, tmem + kColAHi + 8 * kc, blo, 1u);
          mma_ts(d, tmem + kColALo + 8 * kc, bhi, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&mbar))
                     : "memory");
      }
      ++committed;
    }
    // (4) the next round's loads, in flight while (5) runs
    if (rd + 1 < rounds) gather(rd + 1, a);
    // (5) the previous round's outputs into the owned nodes, while this round's MMAs run
    if (rd >= 1) {
      uint32_t r[32];
      tmem_ld32(lane_addr + (((rd - 1) & 1) ? kColD1 : kColD0), r);
      const int vs = (rd - 1) * kSweepVox + (tid >> 3);
      if (vs < nv) {
        const int own = vown[vs];
        const int nl0 = (own >> 8) - 64;
        const float s = vscale[vs];
#pragma unroll
        for (int lm = 0; lm < 8; ++lm) {
          if (own & (1 << lm)) {
            const int nl = nl0 + corner_dx(lm) + kTileX * (corner_dy(lm) + kTileY * corner_dz(lm));
#pragma unroll
            for (int c = 0; c < 3; ++c) atomicAdd(&acc[(nl * 3 + c) * 8 + lcl], s * __uint_as_float(r[3 * lm + c]));
          }
        }
      }
    }
  }
  if (fail) {
    if (tid == 0) atomicExch(err, 1);
    // bounded with the full limit: wait for the last committed MMAs before freeing their memory
    if (committed > 0) mbar_wait(smem_u32(&mbar), (uint32_t)((committed - 1) & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kSweepCols));
  }
  if (fail) return;
  // owned active interior nodes: the sweep's epilogue
  double d1 = 0.0, d2 = 0.0;
  for (int nl = tid >> 3; nl < 128; nl += 16) {
    const int lx = nl % kTileX, ly = (nl / kTileX) % kTileY, lz = nl / (kTileX * kTileY);
    const int x = t.x0 + lx, yv = t.y0 + ly, z = t.z0 + lz;
    if (x > hi_x || yv > hi_y || z > hi_z) continue;
    const int64_t node = node_index(D, x, yv, z);
    if (!(flags[node] & kNodeActive)) continue;  // void node: not written
    const int64_t k0 = vec_index(node, 0, lc);
    float ku[3], v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) ku[c] = (float)(D.scale * (double)acc[(nl * 3 + c) * 8 + lcl]);
    if (MODE == kTcApply) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        v[c] = scale * ku[c];
        d1 += (double)__ldg(u + k0 + c * kNLC) * (double)v[c];
      }
    } else {
      float bc[3], res[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        bc[c] = __ldg(b + k0 + c * kNLC);
        res[c] = bc[c] - ku[c];
      }
      if (MODE == kTcRes) {
#pragma unroll
        for (int c = 0; c < 3; ++c) v[c] = res[c];
      } else {
        float dz[3];
        block_jacobi(binv, node, omega, res, dz);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          v[c] = __ldg(u + k0 + c * kNLC) + dz[c];
          d1 += (double)v[c] * (double)v[c];
          d2 += (double)v[c] * (double)bc[c];
        }
      }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) y[k0 + c * kNLC] = v[c];
  }
  if (MODE == kTcApply || MODE == kTcPost) {
    const int64_t col = (int64_t)t.dom * kNLC + lc;
    const double s1 = block_sum_lc<double>(d1, red);
    if (threadIdx.x < 8) atomicAdd(acc1 + col, s1);
    if (MODE == kTcPost) {
      __syncthreads();
      const double s2 = block_sum_lc<double>(d2, red);
      if (threadIdx.x < 8) atomicAdd(acc2 + col, s2);
    }
  }
}

int allow_sweep_tc(std::string& msg) {
  DTC_CUDA(cudaFuncSetAttribute(k_sweep_tc<kTcApply>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSweepSmem));
  DTC_CUDA(cudaFuncSetAttribute(k_sweep_tc<kTcRes>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSweepSmem));
  DTC_CUDA(cudaFuncSetAttribute(k_sweep_tc<kTcPost>, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::kSweepSmem));
  return DTC_OK;
}

void launch_sweep_tc(int mode, const Tile* tiles, int64_t ntiles, const DomDev* doms, const float* svox,
                     const uint8_t* flags, const float* binv, const float* b, const float* u, float* y, float scale,
                     float omega, double* acc1, double* acc2, const int* dom_active, int* err, cudaStream_t s) {
  if (ntiles <= 0) return;
  const unsigned grid = (unsigned)(3 * ntiles);
  if (mode == kTcApply)
    k_sweep_tc<kTcApply><<<grid, 128, tc::kSweepSmem, s>>>(tiles, doms, svox, flags, binv, b, u, y, scale, omega,
                                                            acc1, acc2, dom_active, err);
  else if (mode == kTcRes)
    k_sweep_tc<kTcRes><<<grid, 128, tc::kSweepSmem, s>>>(tiles, doms, svox, flags, binv, b, u, y, scale, omega, acc1,
                                                          acc2, dom_active, err);
  else
    k_sweep_tc<kTcPost><<<grid, 128, tc::kSweepSmem, s>>>(tiles, doms, svox, flags, binv, b, u, y, scale, omega,
                                                           acc1, acc2, dom_active, err);
}

// Host: build the split Khat in the canonical B layout and upload it.
int upload_tc_operand(const double* khat, cudaStream_t s, std::string& msg) {
  using namespace tc;
  float img[6 * kN * kKc];
  for (int i = 0; i < 6 * kN * kKc; ++i) img[i] = 0.0f;
  for (int n = 0; n < 24; ++n)
    for (int k = 0; k < kK; ++k) {
      const float full = (float)khat[n + 24 * k];
      // round to tf32 (10-bit mantissa, nearest, ties away) on the host
      uint32_t b;
      std::memcpy(&b, &full, 4);
      uint32_t hb = (b + 0x1000u) & 0xFFFFE000u;
      float hi;
      std::memcpy(&hi, &hb, 4);
      float rem = full - hi;
      uint32_t rb;
      std::memcpy(&rb, &rem, 4);
      uint32_t lb = (rb + 0x1000u) & 0xFFFFE000u;
      float lo;
      std::memcpy(&lo, &lb, 4);
      const int kc = k >> 3, kk = k & 7;
      img[(kc * kBChunkBytes + canon_offset(n, kk)) / 4] = hi;
      img[((3 + kc) * kBChunkBytes + canon_offset(n, kk)) / 4] = lo;
    }
  DTC_CUDA(cudaMemcpyToSymbolAsync(c_bsplit, img, sizeof(img), 0, cudaMemcpyHostToDevice, s));
  return DTC_OK;
}

// -------------------------------------------------------------------------------------
// HEX20: the 60x60 element contraction of the brick kernel (ebe.cuh) on the tensor cores.
namespace tc20 {
constexpr int kRows = 128, kVoxPerRound = 32, kLcg = 4;
constexpr int kK = 64, kN = 64, kKc = 8, kChunks = kK / kKc;
constexpr int kBChunkBytes = kN * kKc * 4;      // 2 KB
constexpr int kBx = 4, kBy = 4, kBz = 2;        // brick (voxels)
constexpr int kOx = 2 * kBx, kOy = 2 * kBy, kOz = 2 * kBz;
constexpr int kIx = kOx + 3, kIy = kOy + 3, kIz = kOz + 3;   // staged input nodes (1-voxel halo below)
constexpr int kMaxVox = (kBx + 1) * (kBy + 1) * (kBz + 1);
constexpr uint32_t kColAHi = 0, kColALo = 64, kColD0 = 128, kColD1 = 192;
constexpr uint32_t kTmemCols = 256;
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kN >> 3) << 17) |
                            ((uint32_t)(kRows >> 4) << 24);
// shared memory: B hi/lo (canonical chunks), staged inputs, owned accumulators
constexpr size_t kSmemB = 2 * kChunks * kBChunkBytes;                    // 32 KB
constexpr size_t kSmemIn = (size_t)kIx * kIy * kIz * 3 * kLcg * 4;       // 39.7 KB
constexpr size_t kSmemAcc = (size_t)kOx * kOy * kOz * 3 * kLcg * 4;      // 12 KB
constexpr size_t kSmem = kSmemB + kSmemIn + kSmemAcc + 1024;             // + alignment slack

__device__ constexpr int8_t kRing[20][3] = {
    {0, 0, 0}, {1, 0, 0}, {2, 0, 0}, {2, 1, 0}, {2, 2, 0}, {1, 2, 0}, {0, 2, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 1},
    {2, 2, 1}, {0, 2, 1}, {0, 0, 2}, {1, 0, 2}, {2, 0, 2}, {2, 1, 2}, {2, 2, 2}, {1, 2, 2}, {0, 2, 2}, {0, 1, 2}};

__device__ __forceinline__ void mma_ts(uint32_t tmem_d, uint32_t tmem_a, uint64_t db, uint32_t accumulate) {
  uint32_t z = 0;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "r"(tmem_a), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}
}  // namespace tc20

// y = scale * K u on the owned interior nodes of one brick (HEX20, FP32); DOT: acc += u . y.
// One CTA = one brick of 4 x 4 x 2 voxels (owned nodes 8 x 8 x 4 on the doubled grid) x 4 load
// cases.  The brick's input nodes (with a 1-voxel halo below) are staged in shared memory once;
// per round the 128 rows of A are 32 kept voxels x 4 load cases: each thread reads its voxel's
// 60 DOFs of its load case from the staged nodes, splits them into tf32 hi + lo and stores them
// in its own tensor-memory lane (columns 0-63 hi, 64-127 lo; K padded to 64).  One thread issues
// D = A_hi B_hi + A_hi B_lo + A_lo B_hi (B = the unit element matrix, split on the host, N = 60
// padded to 64) as 24 tcgen05.mma (M 128, N 64, K 8) into one of two 64-column accumulators;
// meanwhile every thread scales the previous round's row by the voxel's modulus factor and adds
// the outputs of owned nodes into shared accumulators, which are written once at the end.
// bsplit: the element matrix split into tf32 hi / lo in the canonical B layout (2 x 8 chunks).
template <bool DOT>
__global__ void __launch_bounds__(128, 2)
    k_ebe_tc(const Tile* __restrict__ bricks, const DomDev* __restrict__ doms, const float* __restrict__ svox,
             const uint8_t* __restrict__ flags, const float* __restrict__ bsplit, const float* __restrict__ u,
             float* __restrict__ y, double scale, double* __restrict__ acc_pw, const int* __restrict__ dom_active,
             int* __restrict__ err) {
  using namespace tc20;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* sB = base;
  float* sin = reinterpret_cast<float*>(base + kSmemB);
  float* sacc = reinterpret_cast<float*>(base + kSmemB + kSmemIn);
  __shared__ int vlist[kMaxVox];      // staged-grid origin of the voxel (its node 0), packed
  __shared__ float vscale[kMaxVox];
  __shared__ int vown[kMaxVox];       // owned ring nodes (20 bits)
  __shared__ int wcount[4];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base;
  __shared__ int fail;
  __shared__ double red[kLcg];

  const Tile t = bricks[blockIdx.x / (kNLC / kLcg)];
  if (dom_active && !dom_active[t.dom]) return;
  const DomDev D = doms[t.dom];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = blockIdx.x % (kNLC / kLcg);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(&tmem_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    fail = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc::smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  if (tid < kLcg) red[tid] = 0.0;
#pragma unroll 4
  for (int i = tid; i < (int)(kSmemB / 16); i += 128)
    reinterpret_cast<float4*>(sB)[i] = __ldg(reinterpret_cast<const float4*>(bsplit) + i);
  for (int i = tid; i < kOx * kOy * kOz * 3 * kLcg; i += 128) sacc[i] = 0.0f;
  // staged input nodes: fine coordinates 2 (x0 - 1) .. 2 (x0 + 4), and likewise in y, z
  const int ix0 = 2 * (t.x0 - 1), iy0 = 2 * (t.y0 - 1), iz0 = 2 * (t.z0 - 1);
  // (the 4 load cases of one (node, component) are 16 contiguous bytes: one vector load)
#pragma unroll 4
  for (int i = tid; i < kIx * kIy * kIz * 3; i += 128) {
    const int c = i % 3, nl = i / 3;
    const int gx = ix0 + nl % kIx, gy = iy0 + (nl / kIx) % kIy, gz = iz0 + nl / (kIx * kIy);
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx < D.n[0] && gy < D.n[1] && gz < D.n[2])
      v = __ldg(reinterpret_cast<const float4*>(u + vec_index(node_index(D, gx, gy, gz), c, g * kLcg)));
    reinterpret_cast<float4*>(sin)[i] = v;
  }

  // kept voxels touching the owned nodes (brick plus a 1-voxel halo below), x-fastest order,
  // with the staged-grid index of their node 0 and the mask of their owned ring nodes
  const int L0 = D.L[0], L1 = D.L[1], L2 = D.L[2];
  const int hx = D.n[0] - 2, hy = D.n[1] - 2, hz = D.n[2] - 2;
  int nv = 0;
  {
    const int q = tid;
    int code = -1, own = 0;
    float sv = 0.0f;
    if (q < kMaxVox) {
      const int qx = q % (kBx + 1), qy = (q / (kBx + 1)) % (kBy + 1), qz = q / ((kBx + 1) * (kBy + 1));
      const int vx = t.x0 - 1 + qx, vy = t.y0 - 1 + qy, vz = t.z0 - 1 + qz;
      if (vx >= 0 && vy >= 0 && vz >= 0 && vx < L0 && vy < L1 && vz < L2) {
        sv = __ldg(svox + D.vox_off + vx + (int64_t)L0 * (vy + (int64_t)L1 * vz));
        if (sv != 0.0f) {
          code = (2 * qx) + kIx * ((2 * qy) + kIy * (2 * qz));
#pragma unroll
          for (int a = 0; a < 20; ++a) {
            const int ox = 2 * vx + kRing[a][0], oy = 2 * vy + kRing[a][1], oz = 2 * vz + kRing[a][2];
            const int lx = ox - 2 * t.x0, ly = oy - 2 * t.y0, lz = oz - 2 * t.z0;
            if (lx >= 0 && lx < kOx && ly >= 0 && ly < kOy && lz >= 0 && lz < kOz && ox >= 1 && ox <= hx &&
                oy >= 1 && oy <= hy && oz >= 1 && oz <= hz)
              own |= 1 << a;
          }
        }
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, code >= 0);
    if (lane == 0) wcount[warp] = __popc(m);
    __syncthreads();
    int off = 0;
    for (int w2 = 0; w2 < warp; ++w2) off += wcount[w2];
    if (code >= 0) {
      const int pos = off + __popc(m & ((1u << lane) - 1));
      vlist[pos] = code;
      vscale[pos] = sv;
      vown[pos] = own;
    }
    nv = wcount[0] + wcount[1] + wcount[2] + wcount[3];
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // B visible to the tensor cores
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t sB_addr = tc::smem_u32(sB);
  const int l = tid & (kLcg - 1);
  const int rounds = (nv + kVoxPerRound - 1) / kVoxPerRound;
  const long long lim = g_tc_spin_limit;
  // staged-grid offset of ring node a relative to the voxel's node 0
  auto ring_off = [](int a) { return kRing[a][0] + kIx * (kRing[a][1] + kIy * kRing[a][2]); };

  int committed = 0;
  for (int rd = 0; rd <= rounds; ++rd) {
    // (1) the MMAs of the previous round have finished: A is free, its accumulator is ready
    if (rd >= 1 && !tc::mbar_wait(tc::smem_u32(&mbar), (uint32_t)((rd - 1) & 1), lim)) atomicOr(&fail, 1);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // (2) this round's A row: the voxel's 60 DOFs of this thread's load case, hi then lo
    if (rd < rounds) {
      const int vs = rd * kVoxPerRound + (tid >> 2);
      const int o = vs < nv ? vlist[vs] : -1;
#pragma unroll
      for (int ch = 0; ch < 4; ++ch) {   // K chunks of 16 columns (the last holds 12 DOFs)
        uint32_t hv[16], lv[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int k = 16 * ch + j;
          float v = 0.0f;
          if (k < 60 && o >= 0) v = sin[((o + ring_off(k / 3)) * 3 + k % 3) * kLcg + l];
          const uint32_t hb = __float_as_uint(v) & 0xFFFFE000u;
          hv[j] = hb;
          lv[j] = __float_as_uint(v - __uint_as_float(hb));
        }
        tc::tmem_st16(lane_addr + kColAHi + 16 * ch, hv);
        tc::tmem_st16(lane_addr + kColALo + 16 * ch, lv);
      }
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (fail) break;
    if (rd < rounds) {
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t d = tmem + ((rd & 1) ? kColD1 : kColD0);
#pragma unroll
        for (int kc = 0; kc < kChunks; ++kc) {
          const uint64_t bhi = tc::smem_desc(sB_addr + kc * kBChunkBytes);
          const uint64_t blo = tc::smem_desc(sB_addr + (kChunks + kc) * kBChunkBytes);
          tc20::mma_ts(d, tmem + kColAHi + 8 * kc, bhi, kc > 0 ? 1u : 0u);
          tc20::mma_ts(d, tmem + kColAHi + 8 * kc, blo, 1u);
          tc20::mma_ts(d, tmem + kColALo + 8 * kc, bhi, 1u);
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         tc::smem_u32(&mbar))
                     : "memory");
      }
      ++committed;
    }
    // (3) the previous round's outputs into the owned nodes, while this round's MMAs run
    if (rd >= 1) {
      const int vs = (rd - 1) * kVoxPerRound + (tid >> 2);
      const bool have = vs < nv;
      const int own = have ? vown[vs] : 0;
      const float s = have ? vscale[vs] : 0.0f;
      // owned-node index of the voxel's node 0: staged origin minus the owned grid's offset (2, 2, 2)
      int on0 = 0;
      if (have) {
        const int o = vlist[vs];
        const int ox = o % kIx, oy = (o / kIx) % kIy, oz = o / (kIx * kIy);
        on0 = (ox - 2) + kOx * ((oy - 2) + kOy * (oz - 2));
      }
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        uint32_t r[32];
        tc::tmem_ld32(lane_addr + ((((rd - 1) & 1) ? kColD1 : kColD0) + 32 * half), r);
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int n = 32 * half + j;
          if (n >= 60) continue;
          const int a = n / 3, c = n % 3;
          if (own & (1 << a)) {
            const int on = on0 + kRing[a][0] + kOx * (kRing[a][1] + kOy * kRing[a][2]);
            atomicAdd(&sacc[(on * 3 + c) * kLcg + l], s * __uint_as_float(r[j]));
          }
        }
      }
    }
  }
  if (fail) {
    if (tid == 0) atomicExch(err, 1);
    // bounded with the full limit: wait for the last committed MMAs before freeing their memory
    if (committed > 0) tc::mbar_wait(tc::smem_u32(&mbar), (uint32_t)((committed - 1) & 1));
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
  }
  if (fail) return;
  // owned active interior nodes: y = scale * acc (once), dot with u
  double dot = 0.0;
  for (int i = tid; i < kOx * kOy * kOz * kLcg; i += 128) {
    const int on = i / kLcg;   // i % kLcg == l: the stride 128 is a multiple of kLcg
    const int lx = on % kOx, ly = (on / kOx) % kOy, lz = on / (kOx * kOy);
    const int gx = 2 * t.x0 + lx, gy = 2 * t.y0 + ly, gz = 2 * t.z0 + lz;
    if (gx < 1 || gy < 1 || gz < 1 || gx > hx || gy > hy || gz > hz) continue;
    const int64_t node = node_index(D, gx, gy, gz);
    if (!(flags[node] & kNodeActive)) continue;
    const int64_t b = vec_index(node, 0, g * kLcg + l);
    const int nin = (lx + 2) + kIx * ((ly + 2) + kIy * (lz + 2));
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float v = (float)(scale * D.scale * (double)sacc[(on * 3 + c) * kLcg + l]);
      y[b + c * kNLC] = v;
      if (DOT) dot += (double)sin[(nin * 3 + c) * kLcg + l] * (double)v;
    }
  }
  if (DOT) {
    atomicAdd(&red[l], dot);
    __syncthreads();
    if (tid < kLcg) atomicAdd(acc_pw + (int64_t)t.dom * kNLC + g * kLcg + tid, red[tid]);
  }
}

// Host: the HEX20 unit element matrix (60 x 60, column-major, symmetric) split into tf32 hi / lo
// in the canonical B layout, zero padded to 64 x 64: 2 x 8 chunks of 2 KB.
void build_tc20_operand(const double* k20, float* img) {
  using namespace tc20;
  std::memset(img, 0, kSmemB);
  for (int n = 0; n < 60; ++n)
    for (int k = 0; k < 60; ++k) {
      const float full = (float)k20[n + 60 * k];
      uint32_t b;
      std::memcpy(&b, &full, 4);
      uint32_t hb = (b + 0x1000u) & 0xFFFFE000u;
      float hi;
      std::memcpy(&hi, &hb, 4);
      float rem = full - hi;
      uint32_t rb;
      std::memcpy(&rb, &rem, 4);
      uint32_t lb = (rb + 0x1000u) & 0xFFFFE000u;
      float lo;
      std::memcpy(&lo, &lb, 4);
      const int kc = k >> 3, kk = k & 7;
      img[(kc * kBChunkBytes + tc::canon_offset(n, kk)) / 4] = hi;
      img[((kChunks + kc) * kBChunkBytes + tc::canon_offset(n, kk)) / 4] = lo;
    }
}

size_t tc20_operand_bytes() { return tc20::kSmemB; }

int allow_ebe_tc(std::string& msg) {
  DTC_CUDA(cudaFuncSetAttribute(k_ebe_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc20::kSmem));
  DTC_CUDA(cudaFuncSetAttribute(k_ebe_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc20::kSmem));
  return DTC_OK;
}

void launch_ebe_tc(const Tile* bricks, int64_t nb, const DomDev* doms, const float* svox, const uint8_t* flags,
                   const float* bsplit, const float* u, float* y, double scale, double* acc_pw, const int* dom_active,
                   int* err, cudaStream_t s) {
  if (nb <= 0) return;
  const unsigned grid = (unsigned)((kNLC / tc20::kLcg) * nb);
  if (acc_pw)
    k_ebe_tc<true><<<grid, 128, tc20::kSmem, s>>>(bricks, doms, svox, flags, bsplit, u, y, scale, acc_pw, dom_active,
                                                  err);
  else
    k_ebe_tc<false><<<grid, 128, tc20::kSmem, s>>>(bricks, doms, svox, flags, bsplit, u, y, scale, nullptr,
                                                   dom_active, err);
}

}  // namespace dtc
