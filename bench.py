"""Benchmark: domains/sec of the batched mixed-precision solver vs the plain FP64 solver.

Workload (default): 512 independent HEX08 domains of 32^3 voxels, bone fraction drawn per
domain from U(0.10, 0.40), 24 load cases each, seeded synthetic volumes (no CT data).
A step = one dtc_solve_batch over the whole batch (mesh, 24 load cases, reactions, 6x6
tensor; the rotation search is not part of the metric step).  Accuracy gate: on a sample
the mixed result must be within 1e-5 (normwise relative) of an FP64 solve at rtol 1e-10.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
import __graft_entry__ as ge  # noqa: E402

METRIC = "domains/sec at ≤1e-5 rel tensor err: mixed+batched vs plain FP64, 1 B200"
TARGET = 1e-5
# rtols tried from loose to tight when an arm calibrates (5, 3, 2, 1 per decade): each arm runs at
# the loosest one whose tensors stay within TARGET / 2 of an FP64 rtol-1e-10 solve on a sample
LADDER = [float(f"{m}e-{k}") for k in range(3, 10) for m in (5, 3, 2, 1)][3:]
# rtol at which the reference algorithm (reaction projection, FP64) meets TARGET/2 on this
# workload: what the plain FP64 GPU arm calibrates to on the 512 x 32^3 batch (5e-7, measured);
# the host-only reference arm cannot calibrate itself
REF_RTOL = 5e-7
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) per algorithmic byte of the fine
# sweeps, measured on 16 domains of 32^3 (profiles/k_matvec_k_mg_matvec_f32_16x32cubed.md: the
# voxel-outer sweeps at their tuned 6 or 8 CTAs per SM; below 1 where part of the input vector
# was still in L2)
DRAM_PER_ALGORITHMIC_BYTE = {"matvec_f32": 0.46, "mg_residual_f32": 0.97, "mg_postsmooth_f32": 1.01}
# FP32 SIMT FMA peak, nominal: 148 SMs x 128 lanes x 2 flop x 1.965 GHz (the sweeps run on the
# FMA pipe, not on tensor cores; the measured peaks cover HBM and bf16 tensor only)
FP32_NOMINAL_TFLOPS = 74.4


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--ndom", type=int, default=None,
                   help="domains per GPU (default: 512; c2 256, c3 2000, c4 64)")
    p.add_argument("--L", type=int, default=32)
    p.add_argument("--rtol", type=float, default=0.0, help="0: calibrate per arm to the accuracy target")
    p.add_argument("--estimator", default="energy", choices=["energy", "reaction"])
    p.add_argument("--precond", default="mg", choices=["mg", "block", "jacobi"],
                   help="preconditioner of the FP32 inner solve of the mixed arm")
    p.add_argument("--matvec", default="auto", choices=["simt", "tensor", "auto"],
                   help="HEX08 fine-level sweeps of the mixed arm: SIMT FP32, tcgen05 (3xTF32), or auto "
                        "(the library times both on the batch and keeps the faster)")
    p.add_argument("--device-mesher", action="store_true",
                   help="mixed arm: mesh the domains on the device (dtc_options.device_mesher)")
    p.add_argument("--max-it", type=int, default=20000)
    p.add_argument("--check", type=int, default=16, help="domains re-solved in FP64 at 1e-10 for the accuracy gate")
    p.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison run")
    p.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    p.add_argument("--profile-step", action="store_true",
                   help="one warm-up and one timed-free mixed solve only (for ncu captures)")
    p.add_argument("--elem", type=int, default=8, choices=[8, 20], help="element type of --profile-step")
    p.add_argument("--config", default="c1", choices=["c0", "c1", "c2", "c3", "c4", "me2"],
                   help="c1 (default): the headline line; c0/c2/c3/c4 print their own measurement lines")
    a = p.parse_args()
    if a.ndom is None:
        a.ndom = {"c2": 256, "c3": 2000, "c4": 64, "me2": 128}.get(a.config, 512)
    return a


def workload(args):
    return {"workload": f"{args.ndom}x{args.L}^3 HEX08 domains per GPU, 24 load cases, BV/TV U(0.10,0.40), "
                        "per-voxel E from gray values",
            "l2": "inputs larger than L2 (vectors are GBs)", "parallelism": f"replicas{args.gpus}"}


def reduce_over_ranks(vals, op="max", device="cuda"):
    """Element-wise max (or min) of a list of floats over all ranks; identity on one process."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in vals]
    t = torch.tensor([float(v) for v in vals], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.MIN)
    return [float(v) for v in t.tolist()]


def make_inputs(dtc, ndom, L, rank=0):
    syn = dtc.synth
    rng = np.random.default_rng(syn.seed_for(1, 10_000 + rank))
    bvtv = rng.uniform(0.10, 0.40, size=ndom)
    grays = [syn.bone_volume((L, L, L), float(bvtv[i]), syn.seed_for(1, rank * ndom + i)) for i in range(ndom)]
    return grays, bvtv


class Clocks:
    """nvidia-smi sampling during the timed region (sm clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) > 8:
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def cpu_baseline(args, dtc, grays, rtol, gpu_res=None):
    """The FP64 CPU oracle on a bounded sample of the same workload: one domain per host
    thread, the first domains of the GPU batch.  With gpu_res (the timed arm's results of the
    same domains) it also reports their largest relative tensor difference from the oracle."""
    orc = ge.load_oracle()
    syn = dtc.synth
    cores = os.cpu_count() or 1
    nsample = min(len(grays), cores, 32)
    doms = [orc.Domain(g, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=rtol, max_it=args.max_it,
                       E_voxel=syn.modulus_of_gray(g)) for g in grays[:nsample]]
    t0 = time.perf_counter()
    ref = orc.solve_batch(doms, nthreads=nsample)
    dt = time.perf_counter() - t0
    out = {"value": nsample / dt, "unit": "domains/s", "cores": nsample, "kind": "port",
           "sample": f"first {nsample} domains of the batch ({args.L}^3, rtol {rtol}), one per thread, "
                     f"{dt:.1f} s"}
    if gpu_res is not None:
        out["max_rel_err_vs_oracle"] = _err(gpu_res[:nsample], ref)
        out["oracle_rtol"] = rtol
        out["oracle_note"] = ("normwise max|C - C_oracle| / max|C_oracle| over the sample; the oracle runs at "
                              "the plain FP64 arm's calibrated rtol, so the figure includes its own solve error")
    return out


def run_reference(args, dtc):
    """The reference's algorithm on the host cores: the FP64 CPU oracle (assembled CSR,
    PETSc-semantics Jacobi-PCG, 24 load cases, homogenisation), one domain per thread."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    orc = ge.load_oracle()
    orc.build()
    syn = dtc.synth
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    nsample = min(args.ndom, cores)   # every host thread it can use, one domain each
    grays, _ = make_inputs(dtc, nsample, args.L)
    rtol = args.rtol if args.rtol > 0 else REF_RTOL
    doms = [orc.Domain(g, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=rtol, max_it=args.max_it,
                       E_voxel=syn.modulus_of_gray(g)) for g in grays]
    times = []
    warm = min(args.warmup, 1)   # a host run needs no device warm-up; bounded total time
    for k in range(warm + args.steps):
        t0 = time.perf_counter()
        orc.solve_batch(doms, nthreads=nsample)
        dt = time.perf_counter() - t0
        if k >= warm:
            times.append(dt)
        if dt > 60:   # bounded: one sample step is enough when the host is slow
            times = times or [dt]
            break
    t = float(np.mean(times))
    v = nsample / t
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "domains/s", "n_gpus": args.gpus,
            "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload(args),
            "cpu_baseline": {"value": v, "unit": "domains/s", "cores": nsample, "kind": "port",
                             "sample": f"{nsample} domains of {args.L}^3 per step, one per thread, rtol {rtol}"},
            "e2e": {"value": v, "unit": "domains/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)



def _timed(fn, steps, warmup):
    """Device time per call (the library's CUDA-event solve time) and host wall time."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    dev, wall = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        d = fn()
        wall.append(time.perf_counter() - t0)
        dev.append(d)
    torch.cuda.synchronize()
    return float(np.mean(dev)), float(np.mean(wall))


def _err(res, truth):
    return max(float(np.abs(r["c"] - t["c"]).max() / np.abs(t["c"]).max()) for r, t in zip(res, truth)
               if r["status"] == 0 and t["status"] == 0)


def run_config(args, dtc):
    """Measurement lines of the other workloads (not the headline metric line)."""
    import torch
    syn = dtc.synth
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    steps, warm = max(1, args.steps), max(1, min(args.warmup, 3))
    line = {"config_id": args.config, "n_gpus": 1, "data": "synthetic"}
    if args.config == "c0":
        # 62^3 volume (60^3 core and a 1-voxel frame), BV/TV 0.25, 27 domains of 20^3, FP64 rtol 1e-10
        vol = syn.bone_volume((62, 62, 62), 0.25, syn.seed_for(0, 0))
        parts = syn.volume_domains(vol, 20)
        doms = [dtc.Domain(sub, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, xa_n=xa, domain_number=d)
                for d, xa, sub in parts]
        with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=True, device=local) as sv:
            def step():
                sv.solve(doms)
                return sv.stats()["ms_solve"]
            dev, wall = _timed(step, steps, warm)
        orc = ge.load_oracle()
        odoms = [orc.Domain(sub, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=1e-10, xa_n=xa, rotation=True)
                 for _, xa, sub in parts]
        cores = min(len(odoms), os.cpu_count() or 1)
        t0 = time.perf_counter()
        ref = orc.solve_batch(odoms, nthreads=cores)
        tcpu = time.perf_counter() - t0
        with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=True, device=local) as sv:
            res = sv.solve(doms)

        def rel(a, b):
            return float(np.abs(a - b).max() / np.abs(b).max())
        line.update({"workload": "27 HEX08 domains of 20^3 from a 62^3 volume (BV/TV 0.25), FP64 rtol 1e-10, "
                                 "rotation search", "gpu_ms_device": dev, "gpu_ms_wall": 1e3 * wall,
                     "gpu_domains_per_s_wall": len(doms) / wall,
                     "cpu_oracle_s": tcpu, "cpu_cores": cores, "cpu_domains_per_s": len(doms) / tcpu,
                     "vs_oracle": {"max_rel_err_c": max(rel(r["c"], t["c"]) for r, t in zip(res, ref)),
                                   "max_rel_err_ff": max(rel(r["ff"], t["ff"]) for r, t in zip(res, ref)),
                                   "max_rel_err_kmacro": max(rel(r["kmacro"], t["kmacro"]) for r, t in zip(res, ref)),
                                   "counts_equal": all((r["ne"], r["nn"], r["nb"]) == (t["ne"], t["nn"], t["nb"])
                                                       for r, t in zip(res, ref)),
                                   "max_abs_iter_diff": int(max(np.abs(r["iters"] - t["iters"]).max()
                                                                for r, t in zip(res, ref)))}})
    elif args.config == "c2":
        # 256 HEX20 domains of 24^3, BV/TV 0.25, mixed vs plain FP64
        n = args.ndom
        grays = [syn.bone_volume((24, 24, 24), 0.25, syn.seed_for(2, i)) for i in range(n)]
        doms = [dtc.Domain(g, elem_type=dtc.HEX20, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA,
                           E_voxel=syn.modulus_of_gray(g)) for g in grays]
        sample = doms[:: max(1, n // 8)]
        with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False, device=local) as ref:
            truth = ref.solve(sample)
        out = {}
        ladder = LADDER
        for arm, kw in (("mixed", dict(precision="mixed", estimator="energy", inner_precond="mg",
                                       mixed_matvec=args.matvec)),
                        ("fp64", dict(precision="fp64", mixed_matvec=args.matvec))):
            # loosest rtol whose tensors stay within TARGET/2 of FP64 at 1e-10 on the sample
            for rt in ladder:
                with dtc.Solver(rtol=rt, rotation_search=False, device=local, **kw) as sv:
                    err = _err(sv.solve(sample), truth)
                if err <= 0.5 * TARGET:
                    break
            with dtc.Solver(rtol=rt, rotation_search=False, device=local, **kw) as sv:

                def step():
                    sv.solve(doms)
                    return sv.stats()["ms_solve"]
                dev, wall = _timed(step, steps, warm)
                tune = {k: round(1e3 * v["ms_total"] / max(v["launches"], 1), 1)
                        for k, v in sv.kernel_stats().items() if k.startswith("autotune_")}
            out[arm] = {"domains_per_s": n / (dev / 1e3), "ms_per_step": dev, "rtol": rt, "max_rel_err": err,
                        "e2e_domains_per_s": n / wall}
            if tune:
                out[arm]["autotune_us_per_fine_application"] = tune
        line.update({"workload": f"{n} HEX20 domains of 24^3, BV/TV 0.25, per-voxel E", "mixed": out["mixed"],
                     "fp64_plain": out["fp64"],
                     "speedup_mixed_over_fp64": out["mixed"]["domains_per_s"] / out["fp64"]["domains_per_s"]})
    elif args.config == "c3":
        # 2000 HEX08 domains, L ~ U{16,24,32,48,64}, BV/TV ~ U(0.05,0.45), mixed + MG, CUDA graphs,
        # rotation search in the step
        n = args.ndom
        rng = np.random.default_rng(syn.seed_for(3, 10_000))
        Ls = rng.choice([16, 24, 32, 48, 64], size=n)
        bv = rng.uniform(0.05, 0.45, size=n)
        grays = [syn.bone_volume((int(L),) * 3, float(b), syn.seed_for(3, i)) for i, (L, b) in enumerate(zip(Ls, bv))]
        doms = [dtc.Domain(g, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, E_voxel=syn.modulus_of_gray(g),
                           domain_number=i) for i, g in enumerate(grays)]
        with dtc.Solver(precision="mixed", rtol=3e-5, rotation_search=True, device=local, estimator="energy",
                        inner_precond="mg", mixed_matvec=args.matvec) as sv:
            res = []

            def step():
                res[:] = sv.solve(doms)
                return sv.stats()["ms_solve"]
            dev, wall = _timed(step, steps, warm)
            kst = sv.kernel_stats()
            rot = kst.get("rotation_search_f64", {})
            tuned = {k[len("autotune_"):]: round(1e3 * v["ms_total"] / max(v["launches"], 1), 1)
                     for k, v in kst.items() if k.startswith("autotune_")}
        sample = [i for i in range(0, n, max(1, n // 12))]
        with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False, device=local) as ref:
            truth = ref.solve([doms[i] for i in sample])
        ok = sum(r["status"] == 0 for r in res)
        line.update({"workload": f"{n} HEX08 domains, L in {{16,24,32,48,64}}, BV/TV U(0.05,0.45), mixed+MG, "
                                 "CUDA-graph CG chunks, rotation search",
                     "domains_per_s_device": n / (dev / 1e3), "domains_per_s_wall": n / wall, "ms_device": dev,
                     "ms_wall": 1e3 * wall, "domains_solved": ok,
                     "max_rel_err_vs_fp64_1e-10": _err([res[i] for i in sample], truth),
                     "rotation_ms": rot.get("ms_total"), "rotation_us_per_domain":
                         1e3 * rot["ms_total"] / n if rot else None,
                     "rotation_fp64_tflops": (rot["flops_per_launch"] * rot["launches"] / (rot["ms_total"] / 1e3)
                                              / 1e12 if rot and rot["ms_total"] > 0 else None),
                     "voxels": int(sum(int(L) ** 3 for L in Ls)),
                     "matvec": args.matvec,
                     "autotune_us_per_launch_summed_over_passes_and_classes": tuned or None})
    elif args.config == "me2":
        # macro order 2 (20-node macro element, 60 load cases): HEX08 domains of 32^3, BV/TV
        # U(0.10, 0.40), per-voxel E; mixed (multigrid, energy estimator over the 60 x 60 Gram
        # matrix of the three column passes) vs plain FP64 (the reference's reaction projection),
        # each at its calibrated rtol; the oracle at rtol 1e-10 on 4 domains
        n = args.ndom
        grays, _ = make_inputs(dtc, n, args.L)
        doms = [dtc.Domain(g, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, E_voxel=syn.modulus_of_gray(g))
                for g in grays]
        sample = doms[:: max(1, n // 8)]
        with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False, device=local, macro_order=2) as ref:
            truth = ref.solve(sample)
        out = {}
        ladder = LADDER
        for arm, kw in (("mixed", dict(precision="mixed", inner_precond="mg", mixed_matvec=args.matvec,
                                       estimator=args.estimator)),
                        ("fp64", dict(precision="fp64", mixed_matvec=args.matvec))):
            for rt in ladder:
                with dtc.Solver(rtol=rt, rotation_search=False, device=local, macro_order=2, **kw) as sv:
                    err = _err(sv.solve(sample), truth)
                if err <= 0.5 * TARGET:
                    break
            with dtc.Solver(rtol=rt, rotation_search=False, device=local, macro_order=2, **kw) as sv:

                def step():
                    sv.solve(doms)
                    return sv.stats()["ms_solve"]
                dev, wall = _timed(step, steps, warm)
            out[arm] = {"domains_per_s": n / (dev / 1e3), "ms_per_step": dev, "rtol": rt, "max_rel_err": err,
                        "e2e_domains_per_s": n / wall}
        orc = ge.load_oracle()
        odoms = [orc.Domain(g, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=1e-10, macro_order=2,
                            E_voxel=syn.modulus_of_gray(g)) for g in grays[:4]]
        t0 = time.perf_counter()
        oref = orc.solve_batch(odoms, nthreads=4)
        tcpu = time.perf_counter() - t0
        with dtc.Solver(precision="mixed", rtol=out["mixed"]["rtol"], rotation_search=False, device=local,
                        macro_order=2, inner_precond="mg", estimator=args.estimator) as sv:
            res = sv.solve(doms[:4])

        def rel(a, b):
            return float(np.abs(a - b).max() / np.abs(b).max())
        line.update({"workload": f"macro order 2 (60 load cases): {n} HEX08 domains of {args.L}^3, "
                                 "BV/TV U(0.10,0.40), per-voxel E", "mixed": out["mixed"], "fp64_plain": out["fp64"],
                     "speedup_mixed_over_fp64": out["mixed"]["domains_per_s"] / out["fp64"]["domains_per_s"],
                     "vs_oracle": {"sample": 4, "oracle_rtol": 1e-10, "oracle_s": tcpu,
                                   "max_rel_err_c": max(rel(r["c"], t["c"]) for r, t in zip(res, oref)),
                                   "max_rel_err_ff": max(rel(r["ff"], t["ff"]) for r, t in zip(res, oref)),
                                   "max_rel_err_kmacro": max(rel(r["kmacro"], t["kmacro"])
                                                             for r, t in zip(res, oref))}})
    elif args.config == "c4":
        # adjoint: 64 HEX08 domains of 48^3, loss ||C - C_target||_F^2, gradient vs one forward solve
        n = args.ndom
        grays = [syn.bone_volume((48, 48, 48), 0.25, syn.seed_for(4, i)) for i in range(n)]
        E = [syn.modulus_of_gray(g) for g in grays]
        doms = [dtc.Domain(g, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, E_voxel=e) for g, e in zip(grays, E)]
        rng = np.random.default_rng(syn.seed_for(4, 99))
        target = np.zeros((n, 6, 6))
        for i in range(n):
            target[i][range(3), range(3)] = rng.uniform(3000, 15000, 3)
            target[i][range(3, 6), range(3, 6)] = rng.uniform(1000, 5000, 3)
        grads = [np.zeros(g.shape, np.float32) for g in grays]
        with dtc.Solver(precision="mixed", rtol=1e-6, rotation_search=False, device=local, estimator="energy",
                        inner_precond="mg", keep_displacements=True) as sv:
            fwd, bwd = [], []
            for k in range(warm + steps):
                t0 = time.perf_counter()
                res = sv.solve(doms)
                t1 = time.perf_counter()
                dc = np.stack([2.0 * (r["c"] - target[i]) for i, r in enumerate(res)])
                sv.energy_grad(dc, grads)
                t2 = time.perf_counter()
                if k >= warm:
                    fwd.append(t1 - t0)
                    bwd.append(t2 - t1)
        # the same step end to end through the torch binding: E a CUDA tensor with requires_grad,
        # C = model(E), loss, backward (moduli in and gradients out through device pointers)
        import importlib
        ag = importlib.import_module(dtc.__name__ + ".autograd")
        model = ag.EffectiveStiffness(grays, precision="mixed", rtol=1e-6, inner_precond="mg", estimator="energy",
                                      device=local)
        Et = torch.tensor(np.stack(E), device=torch.device("cuda", local), requires_grad=True)
        Tt = torch.tensor(target, device=torch.device("cuda", local))
        tf, tb = [], []
        for k in range(warm + steps):
            Et.grad = None
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            C = model(Et)
            loss = ((C - Tt) ** 2).sum()
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            loss.backward()
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            if k >= warm:
                tf.append(t1 - t0)
                tb.append(t2 - t1)
        gmax_t = float(Et.grad.abs().max())
        model.close()
        line.update({"workload": f"adjoint: {n} HEX08 domains of 48^3, BV/TV 0.25, per-voxel E, "
                                 "loss ||C - C_target||_F^2, mixed+MG forward at rtol 1e-6",
                     "forward_s": float(np.mean(fwd)), "adjoint_s": float(np.mean(bwd)),
                     "adjoint_over_forward": float(np.mean(bwd) / np.mean(fwd)),
                     "grad_abs_max": float(max(np.abs(g).max() for g in grads)),
                     "torch_e2e": {"forward_s": float(np.mean(tf)), "backward_s": float(np.mean(tb)),
                                   "backward_over_forward": float(np.mean(tb) / np.mean(tf)),
                                   "grad_abs_max": gmax_t,
                                   "path": "EffectiveStiffness on a CUDA tensor: dtc_solve_batch_device_moduli, "
                                           "dtc_energy_grad_device (no numpy round trip)"}})
    print(json.dumps(line), flush=True)


def share_host_cpus(local, local_world):
    """Pins this rank to its contiguous 1/local_world share of the host CPUs, so the host
    phases of the solver (meshing, packing, multigrid build: one thread per CPU of the
    affinity mask) of the ranks on one node do not oversubscribe it."""
    cpus = sorted(os.sched_getaffinity(0))
    k = len(cpus) // max(local_world, 1)
    if k >= 1 and local_world > 1:
        os.sched_setaffinity(0, cpus[local * k:(local + 1) * k])


def main():
    args = parse()
    dtc = ge.load_package()
    if args.impl == "reference":
        run_reference(args, dtc)
        return
    if args.config != "c1":
        run_config(args, dtc)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
        share_host_cpus(local, int(os.environ.get("LOCAL_WORLD_SIZE", str(world))))
    torch.cuda.set_device(local)
    syn = dtc.synth
    grays, _ = make_inputs(dtc, args.ndom, args.L, rank)
    doms = [dtc.Domain(g, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, E_voxel=syn.modulus_of_gray(g),
                       domain_number=i) for i, g in enumerate(grays)]
    h2d = sum(d.phi.nbytes + d.E_voxel.nbytes for d in doms)
    d2h = args.ndom * 8 * (576 + 36 + 48)

    if args.profile_step:
        # one warm-up solve, then one solve of the mixed arm at --rtol (for ncu launch lists:
        # skip the first launches_per_solve launches)
        rt = args.rtol if args.rtol > 0 else 3e-5
        if args.elem == 20:
            doms = [dtc.Domain(g, elem_type=dtc.HEX20, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA,
                               E_voxel=syn.modulus_of_gray(g)) for g in grays]
        with dtc.Solver(precision="mixed", rtol=rt, max_it=args.max_it, rotation_search=False, device=local,
                        estimator=args.estimator, inner_precond=args.precond, mixed_matvec=args.matvec) as sv:
            sv.solve(doms)
            n0 = sv.stats()["kernel_launches"]
            sv.solve(doms)
            torch.cuda.synchronize()
            print(json.dumps({"profile_step": True, "ndom": args.ndom, "L": args.L, "elem": args.elem, "rtol": rt,
                              "inner_precond": args.precond, "launches_per_solve": n0,
                              "launches_second": sv.stats()["kernel_launches"]}))
        return

    # accuracy gate: both arms are timed at the loosest rtol whose tensors stay within
    # TARGET/2 of an FP64 rtol-1e-10 solve on a sample spread over the batch
    nchk = min(args.check, args.ndom)
    sample = [doms[i] for i in np.linspace(0, args.ndom - 1, nchk).astype(int)]
    with dtc.Solver(precision="fp64", rtol=1e-10, max_it=10 * args.max_it, rotation_search=False, device=local) as ref:
        truth = [r["c"] for r in ref.solve(sample)]

    def max_err(res):
        return max(float(np.abs(r["c"] - t).max() / np.abs(t).max()) for r, t in zip(res, truth))

    ladder = LADDER
    arms = {"mixed": dict(precision="mixed", estimator=args.estimator, inner_precond=args.precond,
                          mixed_matvec=args.matvec),
            "fp64": dict(precision="fp64", estimator="reaction", mixed_matvec=args.matvec)}
    rtol_of, err_of = {}, {}
    for arm, kw in arms.items():
        for rt in ladder if args.rtol <= 0 else [args.rtol]:
            with dtc.Solver(rtol=rt, max_it=args.max_it, rotation_search=False, device=local, **kw) as sv:
                e = max_err(sv.solve(sample))
            if e <= 0.5 * TARGET or args.rtol > 0:
                rtol_of[arm], err_of[arm] = rt, e
                break
        else:
            rtol_of[arm], err_of[arm] = ladder[-1], e

    # every rank times the same configuration: the tightest rtol any rank calibrated
    rtol_of["mixed"], rtol_of["fp64"] = reduce_over_ranks([rtol_of["mixed"], rtol_of["fp64"]], "min")
    mixed = dtc.Solver(precision="mixed", rtol=rtol_of["mixed"], max_it=args.max_it, rotation_search=False,
                       device=local, estimator=args.estimator, inner_precond=args.precond, mixed_matvec=args.matvec,
                       device_mesher=args.device_mesher)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        res = mixed.solve(doms)
    clocks = Clocks(local)
    clocks.start()
    barrier()
    e2e_t, dev_ms = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        res = mixed.solve(doms)
        e2e_t.append(time.perf_counter() - t0)
        dev_ms.append(mixed.stats()["ms_solve"])
    barrier()
    clk = clocks.stop()
    st = mixed.stats()
    step_ms = float(np.mean(dev_ms))
    t_e2e = float(np.mean(e2e_t))
    step_ms, t_e2e = reduce_over_ranks([step_ms, t_e2e], "max")
    value = world * args.ndom / (step_ms / 1e3)
    e2e = world * args.ndom / t_e2e
    idx = np.linspace(0, args.ndom - 1, nchk).astype(int)
    timed_err = max_err([res[i] for i in idx])
    fp64 = None
    if not args.no_fp64:
        with dtc.Solver(precision="fp64", rtol=rtol_of["fp64"], max_it=args.max_it, rotation_search=False,
                        device=local, mixed_matvec=args.matvec) as plain:
            plain.solve(doms)
            fp64_ms = plain.stats()["ms_solve"]
        fp64_ms = reduce_over_ranks([fp64_ms], "max")[0]
        fp64 = {"value": world * args.ndom / (fp64_ms / 1e3), "ms_per_step": fp64_ms, "rtol": rtol_of["fp64"],
                "max_rel_err": err_of["fp64"], "estimator": "reaction (reference)",
                "speedup_mixed_over_fp64": fp64_ms / step_ms}
        # what the precision alone buys: the mixed arm with the plain arm's preconditioner (PETSc-style
        # Jacobi) and estimator, at the loosest rtol that meets the same accuracy gate
        for rt in ladder:
            with dtc.Solver(precision="mixed", rtol=rt, max_it=args.max_it, rotation_search=False, device=local,
                            estimator="reaction", inner_precond="jacobi") as sv:
                ej = max_err(sv.solve(sample))
            if ej <= 0.5 * TARGET:
                break
        rt = reduce_over_ranks([rt], "min")[0]
        with dtc.Solver(precision="mixed", rtol=rt, max_it=args.max_it, rotation_search=False, device=local,
                        estimator="reaction", inner_precond="jacobi") as sv:
            sv.solve(doms)
            mj_ms = sv.stats()["ms_solve"]
        mj_ms = reduce_over_ranks([mj_ms], "max")[0]
        fp64["same_preconditioner"] = {
            "mixed_jacobi_domains_per_s": world * args.ndom / (mj_ms / 1e3), "mixed_jacobi_ms": mj_ms,
            "rtol": rt, "max_rel_err": ej, "speedup_over_fp64_from_precision": fp64_ms / mj_ms,
            "speedup_from_multigrid_and_estimator": mj_ms / step_ms}
    peak, src = measured_peaks()
    # dominant kernel: extra, untimed-for-the-metric steps with CUDA-event timing per launch (the
    # second solve of the handle: one-time allocations and the tuner's timings behind it)
    with dtc.Solver(precision="mixed", rtol=rtol_of["mixed"], max_it=args.max_it, rotation_search=False,
                    device=local, profile_kernels=True, estimator=args.estimator,
                    inner_precond=args.precond, mixed_matvec=args.matvec) as prof:
        prof.solve(doms)
        prof.solve(doms)
        ks = prof.kernel_stats()
    host = {k: ks.pop(k) for k in list(ks) if k.startswith("host_")}   # host phases, wall ms
    tune = {k: ks.pop(k) for k in list(ks) if k.startswith("autotune_")}
    autotune = None
    if tune:
        us = {k[len("autotune_"):]: 1e3 * v["ms_total"] / max(v["launches"], 1) for k, v in tune.items()}
        autotune = {"timed_us_per_launch": us,
                    "pick": "tensor" if us.get("tc_sweep", 1e30) < us.get("simt_sweep", 1e30) else "simt",
                    "note": "simt_sweep / tc_sweep: fine post-smoothing; *_6cta / *_8cta: the SIMT residual, "
                            "post-smoothing and CG-application sweeps at 6 or 8 CTAs per SM; f64_*: the FP64 "
                            "sweep at 4 or 6 CTAs per SM"}
    top = max((k for k in ks if ks[k]["bytes_per_launch"] > 0), key=lambda k: ks[k]["ms_total"])
    kt = ks[top]
    t_launch = kt["ms_total"] / kt["launches"] / 1e3
    achieved = kt["bytes_per_launch"] / t_launch / 1e9
    ratio = DRAM_PER_ALGORITHMIC_BYTE.get(top)
    traffic = kt["bytes_per_launch"] * ratio if ratio else None
    share = {k: round(v["ms_total"] / sum(x["ms_total"] for x in ks.values()), 4) for k, v in ks.items()}
    cpu = (cpu_baseline(args, dtc, grays, rtol_of["fp64"], res) if (rank == 0 and world == 1 and not args.no_cpu)
           else None)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "domains/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
                "config": workload(args),
                "rtol": rtol_of["mixed"], "estimator": args.estimator, "inner_precond": args.precond,
                "matvec": args.matvec, "autotune": autotune, "device_mesher": args.device_mesher,
                "max_rel_err_vs_fp64_1e-10": timed_err, "accuracy_target": TARGET, "accuracy_sample": nchk,
                "fp64_plain": fp64,
                "dof_iterations_per_s": st["dof_iterations"] / (step_ms / 1e3),
                # whole-solver roofline on the streaming model of an FP32 CG iteration: 40 bytes per
                # unconstrained DOF, load case and inner iteration (operator in/out 8 B, CG update 32 B)
                "solver_roofline": {"bytes_per_dof_rhs_iteration": 40,
                                    "achieved_gbs": 40 * st["dof_iterations"] / (step_ms / 1e3) / 1e9,
                                    "peak": peak, "unit": "GB/s",
                                    "frac": 40 * st["dof_iterations"] / (step_ms / 1e3) / 1e9 / peak},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_source": src,
                             "traffic_source": (f"ncu dram bytes / algorithmic bytes = {ratio} on the 16x32^3 case "
                                                "(profiles/k_matvec_k_mg_matvec_f32_16x32cubed.md), scaled to this "
                                                "launch" if ratio else None),
                             "kernel": top, "avg_launch_us": t_launch * 1e6,
                             "flops_per_launch": kt["flops_per_launch"],
                             "achieved_tflops": kt["flops_per_launch"] / t_launch / 1e12,
                             "fp32_fma_frac_of_nominal": kt["flops_per_launch"] / t_launch / 1e12 / FP32_NOMINAL_TFLOPS,
                             "kernel_time_share": share,
                             "host_ms_per_step": {k: v["ms_total"] for k, v in host.items()}},
                "cpu_baseline": cpu,
                "gpu_launches": st["kernel_launches"], "clocks": clk,
                "e2e": {"value": e2e, "unit": "domains/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}}
        print(json.dumps(line), flush=True)
    mixed.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
