"""Oracle results at the benchmarked configurations, for the GPU parity tests.

The oracle (oracle/, FP64 CPU restatement of the reference path, rtol 1e-10) takes minutes
per domain at these sizes, so its results are computed once here and committed as
tests/golden/config_parity.npz; the GPU tests rebuild the same seeded inputs with
dtc_b200.synth and compare against them.  Cases:
  c0 : the 27 HEX08 domains of 20^3 of a 62^3 volume (BV/TV 0.25, constant E), with the
       CR1/CR2 rotation search;
  c1 : 4 HEX08 domains of 32^3 drawn like the headline batch (BV/TV 0.10-0.40, per-voxel E);
  c2 : 4 HEX20 domains of 24^3 (BV/TV 0.25, per-voxel E), the subset of the HEX20 workload.
With --me2 it writes tests/golden/config_parity_me2.npz instead:
  me2: macro order 2 (60 load cases) on the first 4 c0 domains (HEX08, 20^3, constant E) and on
       2 HEX20 domains of 12^3 (per-voxel E).

    python tests/golden/make_config_fixtures.py [--threads N] [--me2]
"""
import argparse
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
import __graft_entry__ as ge  # noqa: E402

OUT = Path(__file__).resolve().parent / "config_parity.npz"
OUT_ME2 = Path(__file__).resolve().parent / "config_parity_me2.npz"


def c0_domains(syn):
    vol = syn.bone_volume((62, 62, 62), 0.25, syn.seed_for(0, 0))
    return syn.volume_domains(vol, 20)


def c1_cases(syn, n=4):
    rng = np.random.default_rng(syn.seed_for(1, 77_000))
    bv = rng.uniform(0.10, 0.40, size=n)
    return [(syn.bone_volume((32, 32, 32), float(bv[i]), syn.seed_for(1, 77_001 + i)), float(bv[i])) for i in range(n)]


def c2_cases(syn, n=4):
    return [syn.bone_volume((24, 24, 24), 0.25, syn.seed_for(2, i)) for i in range(n)]


def me2_hex20_cases(syn, n=2):
    return [syn.bone_volume((12, 12, 12), 0.3, syn.seed_for(2, 900 + i)) for i in range(n)]


def pack(prefix, results, out):
    keys = ("status", "ne", "nn", "nb")
    for k in keys:
        out[f"{prefix}_{k}"] = np.array([r[k] for r in results], np.int64)
    out[f"{prefix}_iters"] = np.stack([r["iters"] for r in results]).astype(np.int64)
    for k in ("c", "ff", "kmacro", "ee"):
        out[f"{prefix}_{k}"] = np.stack([r[k] for r in results])
    if "ang" in results[0]["cr1"]:
        for w in ("cr1", "cr2"):
            out[f"{prefix}_{w}_ang"] = np.stack([r[w]["ang"] for r in results]).astype(np.int64)
            out[f"{prefix}_{w}_jj"] = np.array([r[w]["iters"] for r in results], np.int64)
            for k in ("crit", "angle"):
                out[f"{prefix}_{w}_{k}"] = np.array([r[w][k] for r in results])
            for k in ("n", "aa", "ee"):
                out[f"{prefix}_{w}_{k}"] = np.stack([r[w][k] for r in results])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--me2", action="store_true")
    a = ap.parse_args()
    dtc = ge.load_package()
    orc = ge.load_oracle()
    syn = dtc.synth
    out = {}
    t0 = time.time()
    if a.me2:
        parts = c0_domains(syn)[:4]
        doms = [orc.Domain(sub, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=1e-10, xa_n=xa, macro_order=2)
                for _, xa, sub in parts]
        pack("me2", orc.solve_batch(doms, nthreads=a.threads), out)
        doms = [orc.Domain(g, nen=20, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=1e-10, macro_order=2,
                           E_voxel=syn.modulus_of_gray(g)) for g in me2_hex20_cases(syn)]
        pack("me2h20", orc.solve_batch(doms, nthreads=a.threads), out)
        print(f"me2 done {time.time() - t0:.0f} s", flush=True)
        np.savez_compressed(OUT_ME2, **out)
        print("wrote", OUT_ME2)
        return
    parts = c0_domains(syn)
    doms = [orc.Domain(sub, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=1e-10, xa_n=xa, rotation=True)
            for _, xa, sub in parts]
    pack("c0", orc.solve_batch(doms, nthreads=a.threads), out)
    print(f"c0 done {time.time() - t0:.0f} s", flush=True)
    doms = [orc.Domain(g, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=1e-10, E_voxel=syn.modulus_of_gray(g))
            for g, _ in c1_cases(syn)]
    pack("c1", orc.solve_batch(doms, nthreads=a.threads), out)
    print(f"c1 done {time.time() - t0:.0f} s", flush=True)
    doms = [orc.Domain(g, nen=20, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=1e-10,
                       E_voxel=syn.modulus_of_gray(g)) for g in c2_cases(syn)]
    pack("c2", orc.solve_batch(doms, nthreads=a.threads), out)
    print(f"c2 done {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
