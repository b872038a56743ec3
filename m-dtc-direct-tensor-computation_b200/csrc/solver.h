// solver.h -- device batch solver (kernels.cu) interface used by the C ABI layer.
#pragma once
#include <sched.h>

#include <algorithm>
#include <atomic>
#include <exception>
#include <mutex>
#include <cstdint>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dtc.h"
#include "mesher.h"

namespace dtc {

// Host threads for the per-domain host phases: the requested count, else the CPUs this
// process may run on (its affinity mask, so ranks pinned to disjoint core sets do not
// oversubscribe the node), else the hardware concurrency.
inline int host_thread_count(int requested) {
  if (requested > 0) return requested;
  cpu_set_t set;
  if (sched_getaffinity(0, sizeof(set), &set) == 0) {
    const int n = CPU_COUNT(&set);
    if (n > 0) return n;
  }
  return (int)std::max(1u, std::thread::hardware_concurrency());
}

// Runs f(i) for i in [0, n) on up to `threads` host threads (0: host_thread_count).  An
// exception thrown by f on any thread stops the hand-out of further indices and is rethrown on
// the calling thread once every started thread has joined; if a thread cannot be started, the
// work runs on the threads that could (at least the calling one).
template <class F>
void parallel_for(int64_t n, int threads, F&& f) {
  int nt = host_thread_count(threads);
  nt = (int)std::min<int64_t>(nt, std::max<int64_t>(n, 1));
  std::atomic<int64_t> next(0);
  std::mutex mu;
  std::exception_ptr first;
  auto work = [&]() {
    try {
      for (;;) {
        const int64_t i = next.fetch_add(1);
        if (i >= n) break;
        f(i);
      }
    } catch (...) {
      std::lock_guard<std::mutex> lock(mu);
      if (!first) first = std::current_exception();
      next.store(n);
    }
  };
  std::vector<std::thread> pool;
  try {
    pool.reserve((size_t)nt);
    for (int t = 1; t < nt; ++t) pool.emplace_back(work);
  } catch (...) {   // std::system_error (no thread) or std::bad_alloc: go on with fewer threads
  }
  work();
  for (auto& th : pool) th.join();
  if (first) std::rethrow_exception(first);
}

struct DomainTask {
  const dtc_domain_in* in = nullptr;
  MeshPlan* plan = nullptr;
  dtc_domain_out* out = nullptr;
  int64_t index = 0;          // position in the caller's batch
};

// What a solve keeps for the adjoint: nothing, the displacements on the device (the chunk
// solved last), or a host copy (earlier chunks of a batch split by device memory).
enum KeepMode { kKeepNone = 0, kKeepDevice = 1, kKeepHost = 2 };

struct KernelClass {
  const char* name = "";
  int64_t launches = 0;
  double ms = 0, bytes = 0, flops = 0;   // summed over launches
};

enum KClassId { kcMatvec32, kcMatvec64, kcUpdate32, kcUpdate64, kcDirection32, kcDirection64, kcColstate,
                kcReaction, kcProject, kcMgJacobi, kcMgResidual, kcMgPost, kcMgTransfer, kcMgCoarse,
                kcRotation, kcTuneSimt, kcTuneTc, kcTuneRes4, kcTuneRes5, kcTunePost5, kcTuneApply4, kcTuneApply5,
                kcTuneF64a, kcTuneF64b, kcHostPack, kcHostMgBuild,
                kcNumClasses };   // the last two: host phases (wall ms)

struct SolverStats {
  double ms_solve = 0;   // device time of the solve (CUDA events, inputs resident)
  double ms_wall = 0;    // host wall time of the same section
  double ms_rotation = 0;
  int64_t kernel_launches = 0;
  double dof_iterations = 0;  // sum over domains of free DOFs x load cases x iterations
  KernelClass kc[kcNumClasses];
};

// Host side of one device pass (packed domains, work lists, multigrid plan); kernels.cu.
struct HostBatch;
struct HostBatchDeleter {
  void operator()(HostBatch* p) const;
};
using HostBatchPtr = std::unique_ptr<HostBatch, HostBatchDeleter>;

class DeviceSolver {
 public:
  struct Impl;  // device buffers and stream (kernels.cu)
  DeviceSolver();
  ~DeviceSolver();
  // Bind to a device; returns DTC_OK or an error with msg set.
  int init(int device, std::string& msg);
  // Solve every task (status OK plans only), fill ff/iters/relres of the outputs.
  int solve(std::vector<DomainTask>& tasks, const dtc_options& opt, double nu, std::string& msg);
  // The same in two phases.  prepare: host work only (voxel factors, work lists, multigrid
  // plan), no device state, so it may run on another thread while a solver executes an
  // earlier pass.  solve: the device work of a prepared pass of the same tasks.
  static int prepare(std::vector<DomainTask>& tasks, const dtc_options& opt, double nu, HostBatchPtr& out,
                     std::string& msg);
  int solve(std::vector<DomainTask>& tasks, const dtc_options& opt, double nu, HostBatchPtr batch,
            std::string& msg);
  // Copy a prepared pass's voxel factors to the device through pinned memory on a stream of
  // their own, so that the copy overlaps the solve of the pass before; its solve then waits
  // for the copy instead of uploading them.  Call from one host thread at a time, after
  // prepare and before solve of that pass, while at most one other pass is in flight.  On an
  // error the batch is left as it was (its solve uploads the factors itself).
  int upload_voxels(HostBatch* batch, std::string& msg);
  // Adjoint: dL/dE_voxel for the domains of the last solve (kept displacements).
  // grad_on_device: grad_e[i] are device pointers on this solver's device (filled by device
  // copies, no host round trip); else host pointers.
  int energy_grad(const double* dloss_dc, float* const* grad_e, int64_t n, bool grad_on_device, std::string& msg);
  const SolverStats& stats() const { return stats_; }
  void set_keep(int mode) { keep_ = mode; }
  // Forget what earlier solves kept for the adjoint (start of a batch).
  void clear_kept();

 private:
  Impl* impl_ = nullptr;
  SolverStats stats_;
  int keep_ = kKeepNone;
};

}  // namespace dtc
