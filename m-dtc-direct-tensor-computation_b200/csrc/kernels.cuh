// kernels.cuh -- device helpers shared by the solver kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/dtc.h"
#include "dtc_internal.h"

namespace dtc {

#define DTC_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      msg = std::string(#call) + ": " + cudaGetErrorString(e_);                          \
      return e_ == cudaErrorMemoryAllocation ? DTC_ERR_OUT_OF_MEMORY : DTC_ERR_CUDA;     \
    }                                                                                    \
  } while (0)

// HEX08 local node index (mod_gen_quadmesh.f90:298-306) of voxel corner (cx, cy, cz).
__host__ __device__ constexpr int corner_local(int cx, int cy, int cz) {
  return 4 * cz + (cy ? (cx ? 2 : 3) : (cx ? 1 : 0));
}

// Node index inside a domain and its vector offset.
__device__ __forceinline__ int64_t node_index(const DomDev& D, int x, int y, int z) {
  return D.node_off + x + (int64_t)D.n[0] * (y + (int64_t)D.n[1] * z);
}
__device__ __forceinline__ int64_t vec_index(int64_t node, int c, int lc) {
  return (node * 3 + c) * kNLC + lc;
}

// z = omega * D^-1 r with D^-1 the symmetric 3x3 node-block inverse (00, 11, 22, 01, 02, 12)
__device__ __forceinline__ void block_jacobi(const float* __restrict__ binv, int64_t n, float omega, const float (&r)[3],
                                             float (&z)[3]) {
  const float* b = binv + n * 6;
  const float b0 = __ldg(b), b1 = __ldg(b + 1), b2 = __ldg(b + 2), b3 = __ldg(b + 3), b4 = __ldg(b + 4),
              b5 = __ldg(b + 5);
  z[0] = omega * (b0 * r[0] + b3 * r[1] + b4 * r[2]);
  z[1] = omega * (b3 * r[0] + b1 * r[1] + b5 * r[2]);
  z[2] = omega * (b4 * r[0] + b5 * r[1] + b2 * r[2]);
}

// Epilogues of the tensor-core HEX08 sweep (matvec_tc.cu, launch_sweep_tc)
enum { kTcApply = 0, kTcRes = 1, kTcPost = 2 };

template <typename T>
__device__ __forceinline__ T block_sum_lc(T v, T* smem /* 4 warps x 8 */) {
  // threads with equal (threadIdx.x & 7) carry the same load case
  v += __shfl_xor_sync(0xffffffffu, v, 8);
  v += __shfl_xor_sync(0xffffffffu, v, 16);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane < 8) smem[warp * 8 + lane] = v;
  __syncthreads();
  T s = 0;
  if (threadIdx.x < 8) s = smem[threadIdx.x] + smem[8 + threadIdx.x] + smem[16 + threadIdx.x] + smem[24 + threadIdx.x];
  return s;  // valid in threads 0..7
}

}  // namespace dtc
