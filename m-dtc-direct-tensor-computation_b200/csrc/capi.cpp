// capi.cpp -- the extern "C" boundary (include/dtc.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "../../include/dtc.h"
#include "fe.h"
#include "mesher.h"
#include "solver.h"

struct dtc_handle {
  dtc_options opt;
  dtc::DeviceSolver solver;
  std::string err;
  dtc::SolverStats last;
  float* staging = nullptr;   // pinned host copy of device-resident moduli (dtc_solve_batch_device_moduli)
  size_t staging_n = 0;
  cudaStream_t mesh_stream = nullptr;   // the device mesher's stream (created on first use)
  ~dtc_handle() {
    if (staging) cudaFreeHost(staging);
    if (mesh_stream) cudaStreamDestroy(mesh_stream);
  }
  // meshes in[0..n) on the device into plans; callable from any host thread
  int mesh_on_device(const dtc_domain_in* in, int64_t n, dtc::MeshPlan* plans, bool numbering, std::string& msg) {
    if (cudaSetDevice(opt.device) != cudaSuccess) { msg = "cudaSetDevice failed"; return DTC_ERR_CUDA; }
    if (!mesh_stream && cudaStreamCreateWithFlags(&mesh_stream, cudaStreamNonBlocking) != cudaSuccess) {
      mesh_stream = nullptr;
      msg = "cudaStreamCreate failed";
      return DTC_ERR_CUDA;
    }
    return dtc::mesh_batch_device(in, n, plans, numbering, mesh_stream, msg);
  }
};

namespace {

using namespace dtc;

int validate_domain(const dtc_domain_in& in, std::string& msg) {
  if (in.elem_type != DTC_HEX08 && in.elem_type != DTC_HEX20) { msg = "elem_type must be 8 or 20"; return 1; }
  if (!in.phi) { msg = "phi is NULL"; return 1; }
  if (in.phi_type != 1 && in.phi_type != 2 && in.phi_type != 4) { msg = "phi_type must be 1, 2 or 4"; return 1; }
  for (int d = 0; d < 3; ++d) {
    if (in.L[d] < 1 || in.L[d] > 1024) { msg = "L out of range [1, 1024]"; return 1; }
    if (!(in.delta[d] > 0) || !(in.phdsize[d] > 0)) { msg = "delta and phdsize must be > 0"; return 1; }
  }
  if (in.delta[0] != in.delta[1] || in.delta[0] != in.delta[2]) { msg = "voxels must be cubic (delta equal in x, y, z)"; return 1; }
  if (!(in.E > 0) || !(in.nu > -1.0 && in.nu < 0.5) || !(in.rve_strain != 0)) { msg = "E > 0, -1 < nu < 0.5, rve_strain != 0 required"; return 1; }
  return 0;
}

void plan_all(const dtc_domain_in* in, int64_t n, MeshPlan* plans, bool numbering, int threads) {
  parallel_for(n, threads, [&](int64_t i) { plan_mesh(in[i], numbering, plans[i]); });
}

// The last element kept only by the compaction quirk contributes its 3x3 diagonal block at
// its surviving node; that node is decoupled, so its displacement is the prescribed value
// on the boundary and 0 inside, and its reaction Ke_ll * u enters ff like any other node
// (projected on the 8 or 20 macro shape functions of the macro order).
void quirk_correction(const dtc_domain_in& in, const MeshPlan& mp, double nu, int order, dtc_domain_out* o) {
  if (!mp.last_partial || !mp.last_on_boundary) return;
  const int nen = mp.nen, nd = 3 * nen;
  const int nm = macro_nodes(order), nl = macro_loadcases(order);
  std::vector<double> kh(nd * nd), uu((size_t)nm * 3 * nl);
  voxel_stiffness(nen, nu, kh.data());
  const double a = in.phdsize[0] * in.delta[0];
  const double E = in.E_voxel ? (double)in.E_voxel[mp.last_voxel] : in.E;
  const double s = E * a;
  double x[3], lo[3], hi[3], xi[3], N[20];
  grid_coordinate(in, nen, mp.last_grid, x);
  for (int d = 0; d < 3; ++d) {
    lo[d] = (double)(in.xa_n[d] - 1) * in.delta[d];
    hi[d] = (double)(in.xa_n[d] + in.L[d] - 1) * in.delta[d];
  }
  geom_to_xi(x, lo, hi, xi);
  macro_shape(order, xi, N);
  macro_modes_of_order(order, 1e-6, uu.data());
  double* ff = order == 2 ? o->macro2->ff : o->ff;
  const int ln = mp.last_local;
  for (int lc = 0; lc < nl; ++lc) {
    double g[3], F[3];
    for (int c = 0; c < 3; ++c) g[c] = boundary_value_n(nm, uu.data(), N, c, lc);
    for (int c = 0; c < 3; ++c) {
      F[c] = 0.0;
      for (int cj = 0; cj < 3; ++cj) F[c] += s * kh[(3 * ln + c) + nd * (3 * ln + cj)] * g[cj];
    }
    for (int k = 0; k < 3; ++k)
      for (int l = 0; l < nm; ++l) ff[(k * nm + l) + nl * lc] += F[k] * N[l];
    if (o->displ || o->force) {
      const int64_t id = mp.nn - 1;  // the last node keeps the last id
      for (int c = 0; c < 3; ++c) {
        if (o->displ) o->displ[(size_t)lc * 3 * mp.nn + 3 * id + c] = g[c];
        if (o->force) o->force[(size_t)lc * 3 * mp.nn + 3 * id + c] = F[c];
      }
    }
  }
}

// device bytes per node of a pass: four FP64 and four FP32 nodal vectors and per-node data;
// macro order 2 with the energy estimator keeps two more FP64 solutions (the earlier column passes)
int64_t device_bytes_per_node(const dtc_options& o) {
  return 72 * (4 * 8 + 4 * 4) + 64 + (o.macro_order == 2 && o.tensor_estimator == 1 ? 2 * 72 * 8 : 0);
}

}  // namespace

namespace dtc {
int rotation_search_device(const std::vector<const double*>& ees, std::vector<int64_t>& ang, std::vector<int>& jj,
                           std::vector<double>& crit, cudaStream_t s, int64_t& launches, std::string& msg,
                           double* ms = nullptr);
}

extern "C" {

int32_t dtc_abi_version(void) { return DTC_ABI_VERSION; }

void dtc_default_options(dtc_options* opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->abi_version = DTC_ABI_VERSION;
  opt->precision = DTC_PREC_FP64;
  opt->rtol = 1e-3;       // -ksp_rtol 1.e-03 (f-src/mod_parameters.f90:31)
  opt->max_it = 500000;   // -ksp_max_it 500000 (:32)
  opt->inner_rtol = 0.0;   // automatic: max(0.3 rtol, 1e-7)
  opt->max_refine = 12;
  opt->rotation_search = 1;
  opt->inner_precond = 1;
  opt->device = 0;
}

dtc_status dtc_create(dtc_handle** handle, const dtc_options* opt) {
  if (!handle) return DTC_ERR_INVALID_ARGUMENT;
  *handle = nullptr;
  dtc_options o;
  dtc_default_options(&o);
  if (opt) {
    if (opt->abi_version != DTC_ABI_VERSION) return DTC_ERR_ABI_MISMATCH;
    o = *opt;
  }
  if (!(o.rtol > 0 && o.rtol < 1) || o.max_it < 1 || (o.precision != DTC_PREC_FP64 && o.precision != DTC_PREC_MIXED))
    return DTC_ERR_INVALID_ARGUMENT;
  if (o.inner_precond < 0 || o.inner_precond > 2 || o.mixed_matvec < 0 || o.mixed_matvec > 2 ||
      o.tensor_estimator < 0 || o.tensor_estimator > 1 || o.chunk_domains < 0 || o.graph_chunks < 0 ||
      o.graph_chunks > 1 || o.device_mesher < 0 || o.device_mesher > 1 || o.macro_order < 0 || o.macro_order > 2)
    return DTC_ERR_INVALID_ARGUMENT;
  if (o.macro_order == 0) o.macro_order = 1;
  // macro order 2 has no adjoint (it is derived for the 24 linear load cases)
  if (o.macro_order == 2 && o.keep_displacements != 0) return DTC_ERR_INVALID_ARGUMENT;
  dtc_handle* h = new (std::nothrow) dtc_handle();
  if (!h) return DTC_ERR_OUT_OF_MEMORY;
  h->opt = o;
  int rc = h->solver.init(o.device, h->err);
  if (rc != DTC_OK) { delete h; return (dtc_status)rc; }
  *handle = h;
  return DTC_OK;
}

dtc_status dtc_destroy(dtc_handle* handle) {
  delete handle;
  return DTC_OK;
}

const char* dtc_last_error(const dtc_handle* handle) {
  if (!handle) return "invalid handle";
  return handle->err.c_str();
}

}  // extern "C"

namespace {

// dtc_mesh_out of one planned domain (reference numbering, coordinates, boundary values)
dtc_status fill_mesh_out(const dtc_domain_in* in, const MeshPlan& mp, dtc_mesh_out* out) {
  out->ne = mp.ne; out->nn = mp.nn; out->nb = mp.nb;
  out->status = mp.status;
  out->last_elem_partial = mp.last_partial ? 1 : 0;
  if (mp.status == DTC_DOMAIN_EMPTY || mp.status == DTC_DOMAIN_NO_STRUCTURE) return DTC_OK;
  const int nen = mp.nen;
  if (out->elems) {
    if (out->cap_elems < mp.ne) return DTC_ERR_INVALID_ARGUMENT;
    std::memcpy(out->elems, mp.elems.data(), sizeof(int64_t) * mp.elems.size());
  }
  if (out->macro_order < 0 || out->macro_order > 2) return DTC_ERR_INVALID_ARGUMENT;
  if (out->nodes || out->bnode_ids || out->bnode_vals) {
    if (out->cap_nodes < mp.nn) return DTC_ERR_INVALID_ARGUMENT;
    const int order = out->macro_order == 2 ? 2 : 1;
    const int nm = macro_nodes(order), nl = macro_loadcases(order);
    double lo[3], hi[3];
    std::vector<double> uu((size_t)nm * 3 * nl);
    for (int d = 0; d < 3; ++d) {
      lo[d] = (double)(in->xa_n[d] - 1) * in->delta[d];
      hi[d] = (double)(in->xa_n[d] + in->L[d] - 1) * in->delta[d];
    }
    macro_modes_of_order(order, 1e-6, uu.data());
    int64_t b = 0;
    for (int64_t id = 0; id < mp.nn; ++id) {
      double x[3];
      grid_coordinate(*in, nen, mp.node_grid[id], x);
      if (out->nodes) for (int d = 0; d < 3; ++d) out->nodes[3 * id + d] = x[d];
      if (!grid_on_boundary(in->L, nen, mp.node_grid[id])) continue;
      if (out->bnode_ids) out->bnode_ids[b] = id + 1;
      if (out->bnode_vals) {
        double xi[3], N[20];
        geom_to_xi(x, lo, hi, xi);
        macro_shape(order, xi, N);
        for (int c = 0; c < 3; ++c)
          for (int lc = 0; lc < nl; ++lc)
            out->bnode_vals[lc + nl * (3 * b + c)] = boundary_value_n(nm, uu.data(), N, c, lc);
      }
      ++b;
    }
  }
  return DTC_OK;
}

}  // namespace

extern "C" {

dtc_status dtc_mesh_domain(const dtc_domain_in* in, dtc_mesh_out* out) {
  if (!in || !out) return DTC_ERR_INVALID_ARGUMENT;
  std::string msg;
  if (validate_domain(*in, msg)) return DTC_ERR_INVALID_ARGUMENT;
  MeshPlan mp;
  if (plan_mesh(*in, true, mp) != DTC_OK) return DTC_ERR_INVALID_ARGUMENT;
  return fill_mesh_out(in, mp, out);
}

dtc_status dtc_mesh_batch(dtc_handle* h, const dtc_domain_in* in, int64_t n, dtc_mesh_out* out) {
  if (!h) return DTC_ERR_INVALID_ARGUMENT;
  h->err.clear();
  if (n < 0 || (n > 0 && (!in || !out))) { h->err = "in/out must be non-NULL for n > 0"; return DTC_ERR_INVALID_ARGUMENT; }
  if (n == 0) return DTC_OK;
  bool numbering = false;
  for (int64_t i = 0; i < n; ++i) {
    std::string msg;
    if (validate_domain(in[i], msg)) { h->err = "domain " + std::to_string(i) + ": " + msg; return DTC_ERR_INVALID_ARGUMENT; }
    if (in[i].elem_type != in[0].elem_type) { h->err = "all domains of one call must share elem_type"; return DTC_ERR_INVALID_ARGUMENT; }
    numbering = numbering || out[i].elems || out[i].nodes || out[i].bnode_ids || out[i].bnode_vals;
  }
  std::vector<MeshPlan> plans((size_t)n);
  int rc = h->mesh_on_device(in, n, plans.data(), numbering, h->err);
  if (rc != DTC_OK) return (dtc_status)rc;
  for (int64_t i = 0; i < n; ++i)
    if (dtc_status st = fill_mesh_out(&in[i], plans[i], &out[i])) {
      h->err = "domain " + std::to_string(i) + ": output capacity too small";
      return st;
    }
  return DTC_OK;
}

dtc_status dtc_solve_batch(dtc_handle* h, const dtc_domain_in* in, int64_t n, dtc_domain_out* out) {
  if (!h) return DTC_ERR_INVALID_ARGUMENT;
  h->err.clear();
  if (n < 0 || (n > 0 && (!in || !out))) { h->err = "in/out must be non-NULL for n > 0"; return DTC_ERR_INVALID_ARGUMENT; }
  if (n == 0) return DTC_OK;
  if (cudaSetDevice(h->opt.device) != cudaSuccess) { h->err = "cudaSetDevice failed"; return DTC_ERR_CUDA; }
  for (int64_t i = 0; i < n; ++i) {
    std::string msg;
    if (validate_domain(in[i], msg)) { h->err = "domain " + std::to_string(i) + ": " + msg; return DTC_ERR_INVALID_ARGUMENT; }
    if (in[i].nu != in[0].nu) { h->err = "all domains of one call must share nu"; return DTC_ERR_INVALID_ARGUMENT; }
    if (in[i].elem_type != in[0].elem_type) { h->err = "all domains of one call must share elem_type"; return DTC_ERR_INVALID_ARGUMENT; }
    if (h->opt.macro_order == 2 && !out[i].macro2) {
      h->err = "domain " + std::to_string(i) + ": macro order 2 needs dtc_domain_out.macro2";
      return DTC_ERR_INVALID_ARGUMENT;
    }
  }
  const int order = h->opt.macro_order;
  std::vector<MeshPlan> plans((size_t)n);
  bool want_fields = false;
  for (int64_t i = 0; i < n; ++i) want_fields = want_fields || out[i].displ || out[i].force;
  // Device passes: bounded by 80 % of the free device memory and chunk_domains.  A large batch
  // also starts with a small pass: the host phase of the rest (mesh planning, packing,
  // multigrid plan) runs on host threads while the device solves that first pass.  Every pass
  // repeats the latency-bound tail of the solve (its slowest domain, the coarse levels), so one
  // cut, not more.  Its size f n covers the host phase of the rest, f >= h / (d + h) with a
  // margin of 1.5, for ~1.3 ms of host work per domain and host thread against ~3 ms of device
  // time per domain (32^3 HEX08): f = 0.65 / (T + 0.43) for T host threads, in [1/8, 1/2].
  // The adjoint keeps the last pass on the device: no extra cut with keep_displacements.
  constexpr int64_t kPipelineMin = 256;
  const bool keep = h->opt.keep_displacements != 0;
  const double frac = std::clamp(0.65 / (host_thread_count(h->opt.host_threads) + 0.43), 0.125, 0.5);
  const int64_t pipe = (!keep && n >= kPipelineMin) ? std::max<int64_t>(32, (int64_t)(frac * (double)n)) : 0;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { h->err = "cudaMemGetInfo failed"; return DTC_ERR_CUDA; }
  const double budget = 0.80 * (double)free_b;
  std::vector<int64_t> cuts{0};
  {
    double bytes = 0;
    for (int64_t k = 0; k < n; ++k) {
      const dtc_domain_in& d = in[k];
      const int mg = d.elem_type == DTC_HEX20 ? 2 : 1;   // HEX20 nodes live on the doubled grid
      const double nb = (double)(mg * d.L[0] + 1) * (mg * d.L[1] + 1) * (mg * d.L[2] + 1) * device_bytes_per_node(h->opt);
      const int64_t cnt = k - cuts.back();
      const bool full = (h->opt.chunk_domains > 0 && cnt >= h->opt.chunk_domains) ||
                        (pipe > 0 && cuts.size() == 1 && cnt >= pipe);
      if (k > cuts.back() && (bytes + nb > budget || full)) { cuts.push_back(k); bytes = 0; }
      bytes += nb;
    }
    cuts.push_back(n);
  }
  // host phase of pass c: plans, output headers, solvable tasks, packed batch
  struct Stage {
    std::vector<DomainTask> tasks;
    HostBatchPtr batch;
    int rc = DTC_OK;
    std::string msg;
  };
  auto host_stage_body = [&](size_t c, Stage& st) {
    const int64_t a = cuts[c], b = cuts[c + 1];
    if (h->opt.device_mesher) {
      st.rc = h->mesh_on_device(in + a, b - a, plans.data() + a, want_fields, st.msg);
      if (st.rc != DTC_OK) return;
    } else {
      plan_all(in + a, b - a, plans.data() + a, want_fields, h->opt.host_threads);
    }
    for (int64_t i = a; i < b; ++i) {
      dtc_domain_out* o = &out[i];
      double* keep_d = o->displ;
      double* keep_f = o->force;
      dtc_macro2_out* keep_m = o->macro2;
      std::memset(o, 0, sizeof(*o));
      o->displ = keep_d; o->force = keep_f; o->macro2 = keep_m;
      if (order == 2) std::memset(o->macro2, 0, sizeof(*o->macro2));
      o->domain_number = in[i].domain_number;
      o->status = plans[i].status;
      o->ne = plans[i].ne; o->nn = plans[i].nn; o->nb = plans[i].nb;
      o->n_free_dof = plans[i].n_free_dof;
      if (plans[i].status == DTC_DOMAIN_OK) st.tasks.push_back(DomainTask{&in[i], &plans[i], o, i});
    }
    st.rc = DeviceSolver::prepare(st.tasks, h->opt, in[0].nu, st.batch, st.msg);
    // the voxel factors go to the device now, overlapping the solve of the pass before (the
    // adjoint keeps the buffers of the pass solved last: it uploads with the solve); if the
    // pinned staging cannot be had, the pass uploads them with its solve instead
    if (st.rc == DTC_OK && !keep) {
      std::string ignored;
      h->solver.upload_voxels(st.batch.get(), ignored);
    }
  };
  // the host stage may run on a worker thread: an exception there becomes the pass's status
  auto host_stage = [&](size_t c, Stage& st) {
    try {
      host_stage_body(c, st);
    } catch (const std::bad_alloc&) {
      st.rc = DTC_ERR_OUT_OF_MEMORY;
      st.msg = "host memory exhausted while preparing a device pass";
    } catch (const std::exception& ex) {
      st.rc = DTC_ERR_INTERNAL;
      st.msg = std::string("preparing a device pass: ") + ex.what();
    }
  };
  h->last = SolverStats();
  h->solver.clear_kept();
  std::vector<DomainTask> tasks;
  const size_t npass = cuts.size() - 1;
  Stage cur;
  host_stage(0, cur);
  for (size_t c = 0; c < npass; ++c) {
    Stage next;
    std::thread ahead;
    bool ahead_done = c + 1 >= npass;
    if (!ahead_done) {
      try {
        ahead = std::thread(host_stage, c + 1, std::ref(next));
      } catch (const std::system_error&) {   // no thread: prepare the next pass after this one
      }
    }
    int rc = cur.rc;
    if (rc != DTC_OK) h->err = cur.msg;
    const bool work = rc == DTC_OK && !cur.tasks.empty();
    if (work) {
      // the adjoint keeps the last pass on the device and checkpoints the others to the host
      h->solver.set_keep(!keep ? kKeepNone : (c + 1 == npass ? kKeepDevice : kKeepHost));
      rc = h->solver.solve(cur.tasks, h->opt, in[0].nu, std::move(cur.batch), h->err);
    }
    if (ahead.joinable()) ahead.join();
    else if (!ahead_done && rc == DTC_OK) host_stage(c + 1, next);
    if (rc != DTC_OK) return (dtc_status)rc;
    if (work) {
      const SolverStats& ss = h->solver.stats();
      h->last.ms_solve += ss.ms_solve;
      h->last.ms_wall += ss.ms_wall;
      h->last.kernel_launches += ss.kernel_launches;
      h->last.dof_iterations += ss.dof_iterations;
      for (int q = 0; q < kcNumClasses; ++q) {
        h->last.kc[q].name = ss.kc[q].name;
        h->last.kc[q].launches += ss.kc[q].launches;
        h->last.kc[q].ms += ss.kc[q].ms;
        h->last.kc[q].bytes += ss.kc[q].bytes;
        h->last.kc[q].flops += ss.kc[q].flops;
      }
    }
    tasks.insert(tasks.end(), cur.tasks.begin(), cur.tasks.end());
    cur = std::move(next);
  }
  std::vector<const double*> ees;
  std::vector<dtc_domain_out*> rot_out;
  for (DomainTask& t : tasks) {
    quirk_correction(*t.in, *t.plan, in[0].nu, order, t.out);
    homogenise(order, order == 2 ? t.out->macro2->ff : t.out->ff, t.in->L, t.in->delta, t.in->rve_strain, t.out);
    t.out->density = (double)t.plan->ne / ((double)t.in->L[0] * (double)t.in->L[1] * (double)t.in->L[2]);
    bool finite = true;
    for (int q = 0; q < 36; ++q) finite = finite && std::isfinite(t.out->ee[q]);
    if (h->opt.rotation_search && finite) { ees.push_back(t.out->ee); rot_out.push_back(t.out); }
  }
  if (!ees.empty()) {
    std::vector<int64_t> ang;
    std::vector<int> jj;
    std::vector<double> crit;
    cudaStream_t s = nullptr;
    double ms = 0.0;
    int rc = rotation_search_device(ees, ang, jj, crit, s, h->last.kernel_launches, h->err, &ms);
    if (rc != DTC_OK) return (dtc_status)rc;
    // per candidate about 400 FP64 flops: 2 981 371 sweep points and up to 2 x 16 x 9261 refinements
    KernelClass& kr = h->last.kc[kcRotation];
    kr.name = "rotation_search_f64";
    kr.launches = 2;
    kr.ms = ms;
    double evals = 2981371.0 * (double)ees.size();
    for (int q : jj) evals += 9261.0 * q;
    kr.flops = 400.0 * evals;
    h->last.ms_rotation = ms;
    for (size_t d = 0; d < ees.size(); ++d) {
      finish_rotation(ees[d], 1, &ang[6 * d], jj[2 * d], crit[2 * d], rot_out[d]);
      finish_rotation(ees[d], 2, &ang[6 * d + 3], jj[2 * d + 1], crit[2 * d + 1], rot_out[d]);
    }
  }
  return DTC_OK;
}

dtc_status dtc_solve_batch_device_moduli(dtc_handle* h, const dtc_domain_in* in, int64_t n, dtc_domain_out* out,
                                         const float* const* E_voxel_dev) {
  if (!h) return DTC_ERR_INVALID_ARGUMENT;
  h->err.clear();
  if (n < 0 || (n > 0 && (!in || !out || !E_voxel_dev))) { h->err = "in/out/E_voxel_dev must be non-NULL for n > 0"; return DTC_ERR_INVALID_ARGUMENT; }
  if (n == 0) return DTC_OK;
  if (cudaSetDevice(h->opt.device) != cudaSuccess) { h->err = "cudaSetDevice failed"; return DTC_ERR_CUDA; }
  size_t total = 0;
  for (int64_t i = 0; i < n; ++i)
    if (E_voxel_dev[i]) {
      if (in[i].L[0] < 1 || in[i].L[1] < 1 || in[i].L[2] < 1) { h->err = "L must be >= 1"; return DTC_ERR_INVALID_ARGUMENT; }
      total += (size_t)in[i].L[0] * in[i].L[1] * in[i].L[2];
    }
  if (total > h->staging_n) {
    if (h->staging) cudaFreeHost(h->staging);
    h->staging = nullptr;
    h->staging_n = 0;
    if (cudaMallocHost(&h->staging, sizeof(float) * total) != cudaSuccess) {
      h->staging = nullptr;
      h->err = "cudaMallocHost failed for the moduli staging buffer";
      return DTC_ERR_OUT_OF_MEMORY;
    }
    h->staging_n = total;
  }
  std::vector<dtc_domain_in> loc(in, in + n);
  size_t off = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (!E_voxel_dev[i]) continue;
    const size_t nv = (size_t)in[i].L[0] * in[i].L[1] * in[i].L[2];
    if (cudaMemcpyAsync(h->staging + off, E_voxel_dev[i], sizeof(float) * nv, cudaMemcpyDeviceToHost, nullptr) !=
        cudaSuccess) {
      h->err = "copying the device moduli failed";
      return DTC_ERR_CUDA;
    }
    loc[i].E_voxel = h->staging + off;
    off += nv;
  }
  if (cudaStreamSynchronize(nullptr) != cudaSuccess) { h->err = "copying the device moduli failed"; return DTC_ERR_CUDA; }
  return dtc_solve_batch(h, loc.data(), n, out);
}

dtc_status dtc_rotation_search(dtc_handle* h, const double* ee, int64_t n, dtc_domain_out* out) {
  if (!h) return DTC_ERR_INVALID_ARGUMENT;
  h->err.clear();
  if (n < 0 || (n > 0 && (!ee || !out))) { h->err = "ee/out must be non-NULL for n > 0"; return DTC_ERR_INVALID_ARGUMENT; }
  if (n == 0) return DTC_OK;
  if (cudaSetDevice(h->opt.device) != cudaSuccess) { h->err = "cudaSetDevice failed"; return DTC_ERR_CUDA; }
  std::vector<const double*> ees((size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    ees[i] = ee + 36 * i;
    for (int q = 0; q < 36; ++q)
      if (!std::isfinite(ee[36 * i + q])) { h->err = "tensor " + std::to_string(i) + " is not finite"; return DTC_ERR_INVALID_ARGUMENT; }
  }
  std::vector<int64_t> ang;
  std::vector<int> jj;
  std::vector<double> crit;
  int64_t launches = 0;
  int rc = rotation_search_device(ees, ang, jj, crit, nullptr, launches, h->err);
  if (rc != DTC_OK) return (dtc_status)rc;
  for (int64_t d = 0; d < n; ++d) {
    finish_rotation(ees[d], 1, &ang[6 * d], jj[2 * d], crit[2 * d], &out[d]);
    finish_rotation(ees[d], 2, &ang[6 * d + 3], jj[2 * d + 1], crit[2 * d + 1], &out[d]);
  }
  return DTC_OK;
}

dtc_status dtc_get_kernel_stats(const dtc_handle* h, dtc_kernel_stats* out, int32_t cap, int32_t* count) {
  if (!h || (cap > 0 && !out)) return DTC_ERR_INVALID_ARGUMENT;
  int32_t n = 0;
  for (int c = 0; c < kcNumClasses; ++c) {
    const KernelClass& k = h->last.kc[c];
    if (k.launches == 0) continue;
    if (n < cap) {
      std::memset(&out[n], 0, sizeof(out[n]));
      std::strncpy(out[n].name, k.name, sizeof(out[n].name) - 1);
      out[n].launches = k.launches;
      out[n].ms_total = k.ms;
      out[n].bytes_per_launch = k.bytes / (double)k.launches;
      out[n].flops_per_launch = k.flops / (double)k.launches;
    }
    ++n;
  }
  if (count) *count = n;
  return DTC_OK;
}

dtc_status dtc_element_stiffness(int32_t elem_type, double E, double a, double nu, double* ke) {
  if (!ke || (elem_type != DTC_HEX08 && elem_type != DTC_HEX20) || !(a > 0) || !(nu > -1.0 && nu < 0.5))
    return DTC_ERR_INVALID_ARGUMENT;
  const int nd = 3 * elem_type;
  voxel_stiffness(elem_type, nu, ke);
  for (int i = 0; i < nd * nd; ++i) ke[i] *= E * a;
  return DTC_OK;
}

dtc_status dtc_energy_grad(dtc_handle* h, const double* dloss_dc, float* const* grad_e, int64_t n) {
  if (!h || (n > 0 && (!dloss_dc || !grad_e)) || n < 0) return DTC_ERR_INVALID_ARGUMENT;
  h->err.clear();
  if (!h->opt.keep_displacements) { h->err = "energy_grad needs keep_displacements = 1"; return DTC_ERR_INVALID_ARGUMENT; }
  if (cudaSetDevice(h->opt.device) != cudaSuccess) { h->err = "cudaSetDevice failed"; return DTC_ERR_CUDA; }
  return (dtc_status)h->solver.energy_grad(dloss_dc, grad_e, n, false, h->err);
}

dtc_status dtc_energy_grad_device(dtc_handle* h, const double* dloss_dc, float* const* grad_e_dev, int64_t n) {
  if (!h || (n > 0 && (!dloss_dc || !grad_e_dev)) || n < 0) return DTC_ERR_INVALID_ARGUMENT;
  h->err.clear();
  if (!h->opt.keep_displacements) { h->err = "energy_grad needs keep_displacements = 1"; return DTC_ERR_INVALID_ARGUMENT; }
  if (cudaSetDevice(h->opt.device) != cudaSuccess) { h->err = "cudaSetDevice failed"; return DTC_ERR_CUDA; }
  return (dtc_status)h->solver.energy_grad(dloss_dc, grad_e_dev, n, true, h->err);
}

dtc_status dtc_get_stats(const dtc_handle* h, double* ms_solve, int64_t* kernel_launches, double* dof_iterations) {
  if (!h) return DTC_ERR_INVALID_ARGUMENT;
  if (ms_solve) *ms_solve = h->last.ms_solve;
  if (kernel_launches) *kernel_launches = h->last.kernel_launches;
  if (dof_iterations) *dof_iterations = h->last.dof_iterations;
  return DTC_OK;
}

}  // extern "C"
