// rotation.cu -- parallel rotation search of the 6x6 effective tensor (sm_100a, FP64).
//
// mod_struct_calcmat.f90:533-1603 evaluates, for every candidate rotation (alpha about the
// axis n(phi, eta)) on a 1-degree grid alpha, phi in [0,180], eta in [0,90], the
// off-diagonal energy of B^T E B (CR1: rows 1-4 x cols 5-6; CR2: all 12 upper off-diagonal
// entries), takes the first minimum in column-major order (MINLOC), then refines in a
// +-1 step window at 10x finer resolution until the minimum changes by < 1e-9 or 16 rounds.
// Here one thread evaluates one candidate; a block argmin keeps MINLOC's tie rule (smallest
// linear index, alpha fastest).  This file is compiled with --fmad=false so every
// criterion is evaluated with the same rounding steps as the written expression.
//
// Sines and cosines: the 1-degree sweep reads two tables built on the host, each refinement
// level builds its 3 x 21 values in shared memory; all of them are the correctly rounded
// values (ddmath.h), the same on the host and the device, so the argmin indices do not
// depend on which math library evaluated them.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ddmath.h"
#include "fe.h"
#include "kernels.cuh"
#include "solver.h"

namespace dtc {

__constant__ double c_cosd[181], c_sind[181];

namespace {

constexpr int kSweepA = 181, kSweepP = 181, kSweepE = 91;
constexpr int64_t kSweepN = (int64_t)kSweepA * kSweepP * kSweepE;
constexpr int kSweepBlocks = 64;
constexpr int kRotThreads = 256;

__device__ __forceinline__ void criteria(const double* E, double ca, double sa, double cp, double sp, double ce,
                                         double se, double& c1, double& c2) {
  double n0 = cp * se, n1 = sp * se, n2 = ce;
  const double nr = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
  n0 = n0 / nr; n1 = n1 / nr; n2 = n2 / nr;
  const double omc = 1.0 - ca;
  const double n12 = n0 * n1, n13 = n0 * n2, n23 = n1 * n2;
  const double a11 = ca + n0 * n0 * omc, a22 = ca + n1 * n1 * omc, a33 = ca + n2 * n2 * omc;
  const double a12 = n12 * omc - n2 * sa, a21 = n12 * omc + n2 * sa;
  const double a13 = n13 * omc + n1 * sa, a31 = n13 * omc - n1 * sa;
  const double a23 = n23 * omc - n0 * sa, a32 = n23 * omc + n0 * sa;
  const double s2 = 1.4142135623730951;  // sqrt(2), the value std::sqrt(2.0) rounds to
  double Bm[6][7];  // Bm[r][c] = B(r+1, c), c = 1..6
  Bm[0][1] = a11 * a11; Bm[1][1] = a21 * a21; Bm[2][1] = a31 * a31;
  Bm[3][1] = s2 * a21 * a11; Bm[4][1] = s2 * a11 * a31; Bm[5][1] = s2 * a21 * a31;
  Bm[0][2] = a12 * a12; Bm[1][2] = a22 * a22; Bm[2][2] = a32 * a32;
  Bm[3][2] = s2 * a22 * a12; Bm[4][2] = s2 * a12 * a32; Bm[5][2] = s2 * a22 * a32;
  Bm[0][3] = a13 * a13; Bm[1][3] = a23 * a23; Bm[2][3] = a33 * a33;
  Bm[3][3] = s2 * a23 * a13; Bm[4][3] = s2 * a13 * a33; Bm[5][3] = s2 * a23 * a33;
  Bm[0][4] = s2 * a11 * a12; Bm[1][4] = s2 * a21 * a22; Bm[2][4] = s2 * a31 * a32;
  Bm[3][4] = a21 * a12 + a22 * a11; Bm[4][4] = a11 * a32 + a12 * a31; Bm[5][4] = a21 * a32 + a22 * a31;
  Bm[0][5] = s2 * a11 * a13; Bm[1][5] = s2 * a21 * a23; Bm[2][5] = s2 * a31 * a33;
  Bm[3][5] = a21 * a13 + a23 * a11; Bm[4][5] = a11 * a33 + a13 * a31; Bm[5][5] = a21 * a33 + a23 * a31;
  Bm[0][6] = s2 * a12 * a13; Bm[1][6] = s2 * a22 * a23; Bm[2][6] = s2 * a32 * a33;
  Bm[3][6] = a22 * a13 + a23 * a12; Bm[4][6] = a12 * a33 + a13 * a32; Bm[5][6] = a22 * a33 + a23 * a32;
  // S_j(r) = sum_{c=6..1} B(c,j) E(r,c), then T(i,j) = sum_{r=6..1} B(r,i) S_j(r)
  double S[3][6];
#pragma unroll
  for (int jj = 0; jj < 3; ++jj) {
    const int j = 4 + jj;
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      double s = Bm[5][j] * E[r + 6 * 5];
#pragma unroll
      for (int c = 4; c >= 0; --c) s = s + Bm[c][j] * E[r + 6 * c];
      S[jj][r] = s;
    }
  }
  auto T = [&](int i, int j) {
    const double* Sj = S[j - 4];
    double t = Bm[5][i] * Sj[5];
#pragma unroll
    for (int r = 4; r >= 0; --r) t = t + Bm[r][i] * Sj[r];
    return t;
  };
  const double t14 = T(1, 4), t15 = T(1, 5), t16 = T(1, 6), t24 = T(2, 4), t25 = T(2, 5), t26 = T(2, 6);
  const double t34 = T(3, 4), t35 = T(3, 5), t36 = T(3, 6), t45 = T(4, 5), t46 = T(4, 6), t56 = T(5, 6);
  c1 = t15 * t15 + t16 * t16 + t25 * t25 + t26 * t26 + t35 * t35 + t36 * t36 + t45 * t45 + t46 * t46;
  c2 = t14 * t14 + t15 * t15 + t16 * t16 + t24 * t24 + t25 * t25 + t26 * t26 + t34 * t34 + t35 * t35 + t36 * t36 +
       t45 * t45 + t46 * t46 + t56 * t56;
  if (!(c1 == c1)) c1 = INFINITY;
  if (!(c2 == c2)) c2 = INFINITY;
}

struct ArgMin {
  double v;
  int64_t i;
};
__device__ __forceinline__ bool better(const ArgMin& a, const ArgMin& b) {
  return a.v < b.v || (a.v == b.v && a.i < b.i);
}

__device__ ArgMin block_argmin(ArgMin m, ArgMin* sh) {
  sh[threadIdx.x] = m;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w && better(sh[threadIdx.x + w], sh[threadIdx.x])) sh[threadIdx.x] = sh[threadIdx.x + w];
    __syncthreads();
  }
  ArgMin r = sh[0];
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kRotThreads) k_rot_sweep(const double* __restrict__ ee, ArgMin* __restrict__ part) {
  __shared__ double E[36];
  __shared__ ArgMin sh[kRotThreads];
  const int dom = blockIdx.y;
  if (threadIdx.x < 36) E[threadIdx.x] = ee[(int64_t)dom * 36 + threadIdx.x];
  __syncthreads();
  ArgMin b1{INFINITY, INT64_MAX}, b2{INFINITY, INT64_MAX};
  for (int64_t idx = (int64_t)blockIdx.x * kRotThreads + threadIdx.x; idx < kSweepN;
       idx += (int64_t)gridDim.x * kRotThreads) {
    const int ia = (int)(idx % kSweepA), ip = (int)((idx / kSweepA) % kSweepP), ie = (int)(idx / (kSweepA * kSweepP));
    double c1, c2;
    criteria(E, c_cosd[ia], c_sind[ia], c_cosd[ip], c_sind[ip], c_cosd[ie], c_sind[ie], c1, c2);
    if (c1 < b1.v) { b1.v = c1; b1.i = idx; }
    if (c2 < b2.v) { b2.v = c2; b2.i = idx; }
  }
  const ArgMin r1 = block_argmin(b1, sh);
  const ArgMin r2 = block_argmin(b2, sh);
  if (threadIdx.x == 0) {
    part[((int64_t)dom * kSweepBlocks + blockIdx.x) * 2 + 0] = r1;
    part[((int64_t)dom * kSweepBlocks + blockIdx.x) * 2 + 1] = r2;
  }
}

// One block per (domain, criterion): reduce the sweep, then the x10 refinement loop.
__global__ void __launch_bounds__(kRotThreads) k_rot_refine(const double* __restrict__ ee,
                                                            const ArgMin* __restrict__ part, double pi_div_180,
                                                            int64_t* __restrict__ ang_out, int* __restrict__ jj_out,
                                                            double* __restrict__ crit_out) {
  __shared__ double E[36];
  __shared__ ArgMin sh[kRotThreads];
  __shared__ double tsin[3][21], tcos[3][21];
  const int dom = blockIdx.x, which = blockIdx.y;
  if (threadIdx.x < 36) E[threadIdx.x] = ee[(int64_t)dom * 36 + threadIdx.x];
  ArgMin m{INFINITY, INT64_MAX};
  for (int b = threadIdx.x; b < kSweepBlocks; b += kRotThreads) {
    const ArgMin q = part[((int64_t)dom * kSweepBlocks + b) * 2 + which];
    if (better(q, m)) m = q;
  }
  __syncthreads();
  const ArgMin s0 = block_argmin(m, sh);
  int64_t a[3];
  if (s0.i == INT64_MAX) { a[0] = a[1] = a[2] = 0; }
  else { a[0] = s0.i % kSweepA; a[1] = (s0.i / kSweepA) % kSweepP; a[2] = s0.i / (kSweepA * kSweepP); }
  double prev = s0.v, cur = s0.v;
  double div = pi_div_180;
  int jj = 1;
  for (;;) {
    const int64_t lo[3] = {(a[0] - 1) * 10, (a[1] - 1) * 10, (a[2] - 1) * 10};
    div = div * 0.1;
    if (threadIdx.x < 63) {
      const int d = threadIdx.x / 21, i = threadIdx.x % 21;
      double sv, cv;
      dd::sincos_cr((double)(lo[d] + i) * div, &sv, &cv);
      tsin[d][i] = sv;
      tcos[d][i] = cv;
    }
    __syncthreads();
    ArgMin w{INFINITY, INT64_MAX};
    for (int t = threadIdx.x; t < 21 * 21 * 21; t += kRotThreads) {
      const int i0 = t % 21, i1 = (t / 21) % 21, i2 = t / 441;
      double c1, c2;
      criteria(E, tcos[0][i0], tsin[0][i0], tcos[1][i1], tsin[1][i1], tcos[2][i2], tsin[2][i2], c1, c2);
      const double c = which == 0 ? c1 : c2;
      if (c < w.v) { w.v = c; w.i = t; }
    }
    const ArgMin r = block_argmin(w, sh);
    cur = r.v;
    if (r.i != INT64_MAX) { a[0] = lo[0] + r.i % 21; a[1] = lo[1] + (r.i / 21) % 21; a[2] = lo[2] + r.i / 441; }
    if (fabs(prev - cur) < 1.0e-9 || jj >= 16) break;
    prev = cur;
    jj += 1;
  }
  if (threadIdx.x == 0) {
    int64_t* o = ang_out + ((int64_t)dom * 2 + which) * 3;
    o[0] = a[0]; o[1] = a[1]; o[2] = a[2];
    jj_out[dom * 2 + which] = jj;
    crit_out[dom * 2 + which] = cur;
  }
}

}  // namespace

namespace {
std::mutex g_tables_mu;
bool g_tables_loaded[256] = {false};   // c_cosd / c_sind written on this device ordinal
}  // namespace

// Loads the sweep's degree tables into the current device's constant memory once per device
// and process.  Waits until the copy has landed (a later kernel may run on any stream), so
// the first call must not come inside a stream capture.  Later calls do nothing, so calls
// already in flight on other streams never see the tables being rewritten.
int ensure_degree_tables(std::string& msg) {
  int dev = -1;
  DTC_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) { msg = "device ordinal out of range"; return DTC_ERR_CUDA; }
  std::lock_guard<std::mutex> lock(g_tables_mu);
  if (g_tables_loaded[dev]) return DTC_OK;
  double c[181], sn[181];
  degree_tables(c, sn);
  DTC_CUDA(cudaMemcpyToSymbol(c_cosd, c, sizeof(c)));
  DTC_CUDA(cudaMemcpyToSymbol(c_sind, sn, sizeof(sn)));
  DTC_CUDA(cudaDeviceSynchronize());
  g_tables_loaded[dev] = true;
  return DTC_OK;
}

// Sweep and refinement of every tensor on the device; ms (optional) receives their CUDA-event
// time on stream s.
int rotation_search_device(const std::vector<const double*>& ees, std::vector<int64_t>& ang, std::vector<int>& jj,
                           std::vector<double>& crit, cudaStream_t s, int64_t& launches, std::string& msg,
                           double* ms) {
  const int ndom = (int)ees.size();
  if (ndom == 0) return DTC_OK;
  if (int rc = ensure_degree_tables(msg)) return rc;
  std::vector<double> hee((size_t)36 * ndom);
  for (int d = 0; d < ndom; ++d) std::memcpy(&hee[(size_t)36 * d], ees[d], 36 * sizeof(double));
  double* dee = nullptr;
  ArgMin* dpart = nullptr;
  int64_t* dang = nullptr;
  int* djj = nullptr;
  double* dcrit = nullptr;
  auto cleanup = [&]() {
    cudaFree(dee); cudaFree(dpart); cudaFree(dang); cudaFree(djj); cudaFree(dcrit);
  };
  auto fail = [&](cudaError_t e, const char* what) {
    msg = std::string(what) + ": " + cudaGetErrorString(e);
    cleanup();
    return e == cudaErrorMemoryAllocation ? DTC_ERR_OUT_OF_MEMORY : DTC_ERR_CUDA;
  };
  cudaError_t e;
  if ((e = cudaMalloc(&dee, sizeof(double) * 36 * ndom))) return fail(e, "cudaMalloc");
  if ((e = cudaMalloc(&dpart, sizeof(ArgMin) * 2 * kSweepBlocks * ndom))) return fail(e, "cudaMalloc");
  if ((e = cudaMalloc(&dang, sizeof(int64_t) * 6 * ndom))) return fail(e, "cudaMalloc");
  if ((e = cudaMalloc(&djj, sizeof(int) * 2 * ndom))) return fail(e, "cudaMalloc");
  if ((e = cudaMalloc(&dcrit, sizeof(double) * 2 * ndom))) return fail(e, "cudaMalloc");
  if ((e = cudaMemcpyAsync(dee, hee.data(), sizeof(double) * 36 * ndom, cudaMemcpyHostToDevice, s)))
    return fail(e, "cudaMemcpyAsync");
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if (ms && (cudaEventCreate(&ev[0]) != cudaSuccess || cudaEventCreate(&ev[1]) != cudaSuccess)) ms = nullptr;
  if (ms) cudaEventRecord(ev[0], s);
  k_rot_sweep<<<dim3(kSweepBlocks, ndom), kRotThreads, 0, s>>>(dee, dpart);
  k_rot_refine<<<dim3(ndom, 2), kRotThreads, 0, s>>>(dee, dpart, std::acos(-1.0) / 180.0, dang, djj, dcrit);
  if (ms) cudaEventRecord(ev[1], s);
  launches += 2;
  if ((e = cudaGetLastError())) {
    for (cudaEvent_t q : ev) if (q) cudaEventDestroy(q);
    return fail(e, "rotation kernels");
  }
  ang.resize(6 * ndom); jj.resize(2 * ndom); crit.resize(2 * ndom);
  if ((e = cudaMemcpyAsync(ang.data(), dang, sizeof(int64_t) * 6 * ndom, cudaMemcpyDeviceToHost, s)) ||
      (e = cudaMemcpyAsync(jj.data(), djj, sizeof(int) * 2 * ndom, cudaMemcpyDeviceToHost, s)) ||
      (e = cudaMemcpyAsync(crit.data(), dcrit, sizeof(double) * 2 * ndom, cudaMemcpyDeviceToHost, s)) ||
      (e = cudaStreamSynchronize(s))) {
    for (cudaEvent_t q : ev) if (q) cudaEventDestroy(q);
    return fail(e, "rotation results");
  }
  if (ms) {
    float t = 0.f;
    *ms = cudaEventElapsedTime(&t, ev[0], ev[1]) == cudaSuccess ? (double)t : 0.0;
  }
  for (cudaEvent_t q : ev) if (q) cudaEventDestroy(q);
  cleanup();
  return DTC_OK;
}

// -------------------------------------------------------------------------------------
// Allocation-free variant of the rotation search.  Its only scratch, the per-block sweep
// minima, lives in a file-scope device array sized for kNoAllocMaxDomains domains
// (1024 x 64 blocks x 2 criteria x 16 B = 2 MiB, held by every device that loads the
// library until the process exits).
constexpr int64_t kNoAllocMaxDomains = 1024;
static __device__ __align__(256) ArgMin g_noalloc_part[kNoAllocMaxDomains * kSweepBlocks * 2];

namespace {
std::mutex g_noalloc_mu;
ArgMin* g_noalloc_ptr[256] = {nullptr};   // device address of g_noalloc_part, per device ordinal
}  // namespace

}  // namespace dtc

extern "C" dtc_status dtc_rotation_search_noalloc(const double* ee, int64_t n, int64_t* ang, int32_t* jj,
                                                  double* crit, void* stream) {
  using namespace dtc;
  if (n < 0 || n > kNoAllocMaxDomains) return DTC_ERR_INVALID_ARGUMENT;
  if (n == 0) return DTC_OK;
  if (!ee || !ang || !jj || !crit) return DTC_ERR_INVALID_ARGUMENT;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return DTC_ERR_CUDA;
  ArgMin* part = nullptr;
  {
    // first call on a device: resolve the scratch array's device address and load the
    // degree tables of the sweep, with that device current
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_part) != cudaSuccess || !p) return DTC_ERR_CUDA;
      std::string msg;
      if (ensure_degree_tables(msg) != DTC_OK) return DTC_ERR_CUDA;   // uploads and waits for them
      g_noalloc_ptr[dev] = static_cast<ArgMin*>(p);
    }
    part = g_noalloc_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // every block of the sweep writes its own two minima, so no clearing is needed
  k_rot_sweep<<<dim3(kSweepBlocks, (unsigned)n), kRotThreads, 0, s>>>(ee, part);
  k_rot_refine<<<dim3((unsigned)n, 2), kRotThreads, 0, s>>>(ee, part, std::acos(-1.0) / 180.0, ang, jj, crit);
  return cudaGetLastError() == cudaSuccess ? DTC_OK : DTC_ERR_CUDA;
}
