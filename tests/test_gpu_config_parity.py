"""GPU path vs the oracle at the benchmarked configurations, through the C ABI.

The oracle's FP64 results (rtol 1e-10) for these inputs are committed in
tests/golden/config_parity.npz (made by tests/golden/make_config_fixtures.py, which also
defines the inputs rebuilt here from their seeds):
  c0 : 27 HEX08 domains of 20^3 from a 62^3 volume, constant E, rotation search;
  c1 : 4 HEX08 domains of 32^3 drawn like the headline batch, per-voxel E;
  c2 : 4 HEX20 domains of 24^3, per-voxel E;
and, in tests/golden/config_parity_me2.npz (the same script with --me2), macro order 2 (60 load
cases) on the first 4 c0 domains and on 2 HEX20 domains of 12^3.
Tolerances (normwise relative on C, ff, K_macro): FP64 path 1e-6, mixed path 1e-5.
Counts and indices (ne, nn, nb; rotation argmin indices and refinement depth) must be equal.
"""
import importlib.util

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-6
TOL_MIXED = 1e-5


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN / "config_parity.npz")


@pytest.fixture(scope="module")
def cases(dtc):
    spec = importlib.util.spec_from_file_location("make_config_fixtures", GOLDEN / "make_config_fixtures.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    syn = dtc.synth
    return {"c0": m.c0_domains(syn), "c1": m.c1_cases(syn), "c2": m.c2_cases(syn),
            "me2h20": m.me2_hex20_cases(syn)}


def check_tensors(res, gold, key, tol, counts=True):
    for i, r in enumerate(res):
        assert r["status"] == gold[f"{key}_status"][i] == 0
        if counts:
            assert (r["ne"], r["nn"], r["nb"]) == (gold[f"{key}_ne"][i], gold[f"{key}_nn"][i], gold[f"{key}_nb"][i])
        assert rel(r["c"], gold[f"{key}_c"][i]) <= tol, (key, i, rel(r["c"], gold[f"{key}_c"][i]))
        assert rel(r["ff"], gold[f"{key}_ff"][i]) <= tol
        assert rel(r["kmacro"], gold[f"{key}_kmacro"][i]) <= tol


def test_c0_fp64_matches_oracle(dtc, gold, cases):
    syn = dtc.synth
    doms = [dtc.Domain(sub, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, xa_n=xa, domain_number=d)
            for d, xa, sub in cases["c0"]]
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=True) as s:
        res = s.solve(doms)
    check_tensors(res, gold, "c0", TOL_FP64)
    for i, r in enumerate(res):
        assert r["domain_number"] == cases["c0"][i][0]
        # the same PETSc CG recurrence: iteration counts agree up to where rounding (the order of
        # the dot-product sums, which follows the CTA schedule) moves the crossing of the
        # threshold: measured up to 9 of ~250-340 iterations; allowed 5 %
        assert (np.abs(r["iters"] - gold["c0_iters"][i]) <= np.maximum(3, 0.05 * gold["c0_iters"][i])).all()
        # rotation search on a tensor that differs from the oracle's in the 10th digit (the order of
        # the device's dot-product and reaction sums follows the CTA schedule): the criterion
        # agrees to that level, but where two rotations reach it within rounding the argmin may
        # jump between them, and so may the rotated tensor (measured: 0.9 % on its diagonal for one
        # c0 domain in one of six runs).  The rotated tensor is checked through invariants of the
        # rotation, C_iijj (the sum of the normal block) and the Frobenius norm of the 6x6 (the
        # rotation is orthogonal in the Mandel form), against the unrotated tensor; bit-exact
        # argmin parity on identical tensors is tested in test_rotation_search_bit_exact and
        # test_rotation_c0_indices_from_fixture.
        e2 = np.abs(gold["c0_ee"][i]).max() ** 2
        for w in ("cr1", "cr2"):
            assert abs(r[w]["crit"] - gold[f"c0_{w}_crit"][i]) <= 1e-8 * e2
            assert abs(r[w]["ee"][:3, :3].sum() - gold["c0_ee"][i][:3, :3].sum()) <= 1e-6 * np.abs(gold["c0_ee"][i]).max()
            assert rel(np.linalg.norm(r[w]["ee"]), np.linalg.norm(gold["c0_ee"][i])) <= 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_macro_order2_matches_oracle(dtc, cases, precision):
    """Macro order 2 at c0's domain size (and HEX20 micro elements): C, ff(60 x 60), K_macro."""
    g2 = np.load(GOLDEN / "config_parity_me2.npz")
    syn = dtc.synth
    kw = dict(precision=precision, rotation_search=False, macro_order=2)
    if precision == "mixed":
        kw.update(inner_precond="mg", estimator="energy")
    tol = TOL_FP64 if precision == "fp64" else TOL_MIXED
    doms = [dtc.Domain(sub, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, xa_n=xa) for _, xa, sub in cases["c0"][:4]]
    with dtc.Solver(rtol=1e-10, **kw) as s:
        check_tensors(s.solve(doms), g2, "me2", tol)
    doms = [dtc.Domain(g, elem_type=dtc.HEX20, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA,
                       E_voxel=syn.modulus_of_gray(g)) for g in cases["me2h20"]]
    with dtc.Solver(rtol=1e-10, **kw) as s:
        check_tensors(s.solve(doms), g2, "me2h20", tol)


def test_c1_matches_oracle(dtc, gold, cases):
    syn = dtc.synth
    doms = [dtc.Domain(g, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, E_voxel=syn.modulus_of_gray(g))
            for g, _ in cases["c1"]]
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False) as s:
        check_tensors(s.solve(doms), gold, "c1", TOL_FP64)
    # the headline arm: mixed precision, multigrid inner solve, energy estimator, at the
    # loosest rtol the benchmark calibrates to on this workload
    with dtc.Solver(precision="mixed", rtol=3e-5, rotation_search=False, inner_precond="mg",
                    estimator="energy") as s:
        check_tensors(s.solve(doms), gold, "c1", TOL_MIXED)


def test_c2_hex20_matches_oracle(dtc, gold, cases):
    syn = dtc.synth
    doms = [dtc.Domain(g, elem_type=dtc.HEX20, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA,
                       E_voxel=syn.modulus_of_gray(g)) for g in cases["c2"]]
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False) as s:
        check_tensors(s.solve(doms), gold, "c2", TOL_FP64)
    with dtc.Solver(precision="mixed", rtol=1e-4, rotation_search=False, inner_precond="mg",
                    estimator="energy") as s:
        check_tensors(s.solve(doms), gold, "c2", TOL_MIXED)


def synthetic_tensors():
    """Symmetric 6x6 tensors: rotated orthotropic ones, an isotropic one (flat criterion: every
    candidate ties up to rounding) and a cubic one."""
    rng = np.random.default_rng(4242)
    out = []
    for k in range(3):
        E = rng.uniform(3000, 15000, 3)
        G = rng.uniform(1000, 5000, 3)
        S = np.zeros((6, 6))
        S[range(3), range(3)] = 1 / E
        nu = 0.3
        for i in range(3):
            for j in range(3):
                if i != j:
                    S[i, j] = -nu / E[i]
        S = 0.5 * (S + S.T)
        S[range(3, 6), range(3, 6)] = 1 / (2 * G)   # Mandel (sqrt(2)) shear convention
        out.append(np.linalg.inv(S))
    lam, mu = 5000.0, 3000.0
    iso = np.zeros((6, 6))
    iso[:3, :3] = lam
    iso[range(3), range(3)] += 2 * mu
    iso[range(3, 6), range(3, 6)] = 2 * mu
    out.append(iso)
    cub = iso.copy()
    cub[range(3, 6), range(3, 6)] = 1500.0
    out.append(cub)
    return out


def test_rotation_search_bit_exact(dtc, orc, gold):
    """Argmin indices, refinement depth and criterion equal the oracle's bit for bit when both
    search the same tensor; the derived angle equals it, axis, frame and rotated tensor agree to
    rounding (both use correctly rounded sines and cosines for the search)."""
    ees = list(gold["c0_ee"][:12]) + synthetic_tensors()
    refs = [orc.rotation_search(e) for e in ees]
    with dtc.Solver(precision="fp64", rotation_search=True) as s:
        res = s.rotation_search(np.stack(ees))
    for i, (r, ref) in enumerate(zip(res, refs)):
        for w in ("cr1", "cr2"):
            a, b = r[w], ref[w]
            assert a["iters"] == b["iters"], (i, w, a["iters"], b["iters"])
            assert a["crit"] == b["crit"], (i, w, a["crit"], b["crit"])
            assert a["angle"] == b["angle"], (i, w, a["angle"], b["angle"])
            assert np.abs(a["n"] - b["n"]).max() <= 1e-12
            assert np.abs(a["aa"] - b["aa"]).max() <= 1e-12
            assert rel(a["ee"], b["ee"]) <= 1e-12
    # the raw argmin indices through the allocation-free entry (device in, device out)
    import torch
    lib = dtc.capi.load()
    dev = torch.device("cuda", 0)
    n = len(ees)
    ee_d = torch.tensor(np.stack([e.reshape(-1, order="F") for e in ees]), dtype=torch.float64, device=dev)
    ang = torch.zeros((n, 2, 3), dtype=torch.int64, device=dev)
    jj = torch.zeros((n, 2), dtype=torch.int32, device=dev)
    crit = torch.zeros((n, 2), dtype=torch.float64, device=dev)
    assert lib.dtc_rotation_search_noalloc(ee_d.data_ptr(), n, ang.data_ptr(), jj.data_ptr(), crit.data_ptr(),
                                           None) == dtc.capi.DTC_OK
    torch.cuda.synchronize()
    a, j = ang.cpu().numpy(), jj.cpu().numpy()
    for i, ref in enumerate(refs):
        for w, k in enumerate(("cr1", "cr2")):
            assert (a[i, w] == ref[k]["ang"]).all(), (i, k, a[i, w], ref[k]["ang"])
            assert j[i, w] == ref[k]["iters"]


def test_rotation_c0_indices_from_fixture(dtc, gold):
    """The same check against the committed oracle search of all 27 c0 tensors."""
    with dtc.Solver(precision="fp64", rotation_search=True) as s:
        res = s.rotation_search(gold["c0_ee"])
    for i, r in enumerate(res):
        for w in ("cr1", "cr2"):
            assert r[w]["iters"] == gold[f"c0_{w}_jj"][i]
            assert r[w]["crit"] == gold[f"c0_{w}_crit"][i]
            assert r[w]["angle"] == gold[f"c0_{w}_angle"][i]
            assert rel(r[w]["ee"], gold[f"c0_{w}_ee"][i]) <= 1e-12
