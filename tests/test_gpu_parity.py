"""GPU path vs the FP64 oracle, through the C ABI (include/dtc.h).

Tolerances (normwise relative, max|C - C*| / max|C*|, the judged quantity):
  FP64 path  <= 1e-6 against the oracle at rtol 1e-10,
  mixed path <= 1e-5 against the oracle at rtol 1e-10.
Integer/index outputs (ne, nn, nb, reference DOF numbering) must be identical.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-6
TOL_MIXED = 1e-5


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def make_pair(dtc, orc, shape, bvtv, seed, E_voxel=False, **kw):
    syn = dtc.synth
    gray = syn.bone_volume(shape, bvtv, seed)
    ev = syn.modulus_of_gray(gray) if E_voxel else None
    d = dtc.Domain(gray, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, E_voxel=ev, **kw)
    o = orc.Domain(gray, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=1e-10, E_voxel=ev, **kw)
    return d, o


@pytest.fixture(scope="module")
def batch(dtc, orc):
    pairs = [make_pair(dtc, orc, (12, 12, 12), b, dtc.synth.seed_for(7, i))
             for i, b in enumerate((0.15, 0.25, 0.35, 0.5))]
    pairs.append(make_pair(dtc, orc, (9, 11, 10), 0.4, dtc.synth.seed_for(7, 9)))   # non-cubic box
    pairs.append(make_pair(dtc, orc, (12, 12, 12), 0.3, dtc.synth.seed_for(7, 10), E_voxel=True))
    refs = orc.solve_batch([p[1] for p in pairs])
    return pairs, refs


def test_fp64_matches_oracle(dtc, batch):
    pairs, refs = batch
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False) as s:
        res = s.solve([p[0] for p in pairs])
        st = s.stats()
    assert st["kernel_launches"] > 0
    for r, ref in zip(res, refs):
        assert r["status"] == ref["status"] == 0
        assert (r["ne"], r["nn"], r["nb"]) == (ref["ne"], ref["nn"], ref["nb"])
        assert rel(r["c"], ref["c"]) <= TOL_FP64
        assert rel(r["ff"], ref["ff"]) <= TOL_FP64
        assert rel(r["kmacro"], ref["kmacro"]) <= TOL_FP64
        # same Jacobi-PCG recurrence: iteration counts agree up to rounding near the threshold
        assert np.abs(r["iters"] - ref["iters"]).max() <= 2


@pytest.mark.parametrize("matvec,precond", [("simt", "block"), ("tensor", "block"), ("simt", "jacobi"),
                                            ("simt", "mg"), ("tensor", "mg"), ("tensor", "jacobi")])
def test_mixed_matches_oracle(dtc, batch, matvec, precond):
    pairs, refs = batch
    with dtc.Solver(precision="mixed", rtol=1e-10, rotation_search=False, mixed_matvec=matvec,
                    inner_precond=precond) as s:
        res = s.solve([p[0] for p in pairs])
    for r, ref in zip(res, refs):
        assert r["status"] == 0
        assert rel(r["c"], ref["c"]) <= TOL_MIXED
        assert r["refine_steps"] >= 1


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_energy_estimator_matches_oracle(dtc, batch, precision):
    """ff from the energy products equals the reaction projection at convergence."""
    pairs, refs = batch
    with dtc.Solver(precision=precision, rtol=1e-10, rotation_search=False, estimator="energy") as s:
        res = s.solve([p[0] for p in pairs])
    tol = TOL_FP64 if precision == "fp64" else TOL_MIXED
    for r, ref in zip(res, refs):
        assert rel(r["c"], ref["c"]) <= tol
        assert rel(r["ff"], ref["ff"]) <= tol


def test_fields_in_reference_numbering(dtc, orc):
    d, o = make_pair(dtc, orc, (8, 8, 8), 0.4, dtc.synth.seed_for(7, 20))
    ref = orc.solve_domain(o, with_arrays=True)
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False) as s:
        r = s.solve([d], want_fields=True)[0]
    assert rel(r["displ"], ref["displ"]) <= 1e-7
    assert rel(r["force"], ref["force"]) <= 1e-6


def test_solid_cube_isotropic(dtc):
    E, nu = 5600.0, 0.3
    gray = np.full((6, 6, 6), 14250, np.int16)
    with dtc.Solver(precision="fp64", rtol=1e-12, rotation_search=False) as s:
        r = s.solve([dtc.Domain(gray, E=E, nu=nu, delta=0.01)])[0]
    lam, mu = E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[range(3), range(3)] += 2 * mu
    C[3, 3] = C[4, 4] = C[5, 5] = mu
    assert rel(r["c"], C) < 1e-8


def test_statuses(dtc):
    empty = np.zeros((6, 6, 6), np.int16)
    full = np.full((6, 6, 6), 100, np.int16)
    with dtc.Solver(precision="fp64", rtol=1e-8, rotation_search=False) as s:
        r = s.solve([dtc.Domain(empty, domain_number=3), dtc.Domain(full, domain_number=4)])
    assert r[0]["status"] == dtc.DOMAIN_EMPTY and r[0]["domain_number"] == 3
    assert r[1]["status"] == dtc.DOMAIN_OK and r[1]["domain_number"] == 4
    with dtc.Solver(precision="fp64", rtol=1e-10, max_it=3, rotation_search=False) as s:
        r = s.solve([dtc.Domain(full)])
    assert r[0]["status"] == dtc.DOMAIN_MAX_IT
    assert r[0]["iters"].max() == 3


def test_rotation_matches_oracle(dtc, orc, batch):
    pairs, refs = batch
    d, o = pairs[1]
    o.s.rotation = 1
    ref = orc.solve_domain(o)
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=True) as s:
        r = s.solve([d])[0]
    for k in ("cr1", "cr2"):
        a, b = r[k], ref[k]
        assert abs(a["crit"] - b["crit"]) <= 1e-9 + 1e-6 * abs(b["crit"])
        assert rel(np.diag(a["ee"]), np.diag(b["ee"])) <= 1e-6


# ---------------------------------------------------------------- HEX20 (20-node serendipity bricks)

def make_pair20(dtc, orc, shape, bvtv, seed, E_voxel=False):
    syn = dtc.synth
    gray = syn.bone_volume(shape, bvtv, seed)
    ev = syn.modulus_of_gray(gray) if E_voxel else None
    d = dtc.Domain(gray, elem_type=dtc.HEX20, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, E_voxel=ev)
    o = orc.Domain(gray, nen=20, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=1e-10, E_voxel=ev)
    return d, o


@pytest.fixture(scope="module")
def batch20(dtc, orc):
    pairs = [make_pair20(dtc, orc, (8, 8, 8), b, dtc.synth.seed_for(20, i)) for i, b in enumerate((0.2, 0.4))]
    pairs.append(make_pair20(dtc, orc, (7, 9, 6), 0.45, dtc.synth.seed_for(20, 5)))   # non-cubic box
    pairs.append(make_pair20(dtc, orc, (8, 8, 8), 0.3, dtc.synth.seed_for(20, 6), E_voxel=True))
    refs = orc.solve_batch([p[1] for p in pairs])
    return pairs, refs


def test_hex20_fp64_matches_oracle(dtc, batch20):
    pairs, refs = batch20
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False) as s:
        res = s.solve([p[0] for p in pairs])
    for r, ref in zip(res, refs):
        assert r["status"] == ref["status"] == 0
        assert (r["ne"], r["nn"], r["nb"]) == (ref["ne"], ref["nn"], ref["nb"])
        assert rel(r["c"], ref["c"]) <= TOL_FP64
        assert rel(r["ff"], ref["ff"]) <= TOL_FP64
        assert np.abs(r["iters"] - ref["iters"]).max() <= 2


@pytest.mark.parametrize("precond", ["block", "jacobi", "mg"])
def test_hex20_mixed_matches_oracle(dtc, batch20, precond):
    pairs, refs = batch20
    with dtc.Solver(precision="mixed", rtol=1e-10, rotation_search=False, inner_precond=precond) as s:
        res = s.solve([p[0] for p in pairs])
    for r, ref in zip(res, refs):
        assert r["status"] == 0
        assert rel(r["c"], ref["c"]) <= TOL_MIXED


def test_hex20_fields_in_reference_numbering(dtc, orc):
    d, o = make_pair20(dtc, orc, (6, 6, 6), 0.45, dtc.synth.seed_for(20, 9))
    ref = orc.solve_domain(o, with_arrays=True)
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False) as s:
        r = s.solve([d], want_fields=True)[0]
    assert r["displ"].shape == ref["displ"].shape
    assert rel(r["displ"], ref["displ"]) <= 1e-7
    assert rel(r["force"], ref["force"]) <= 1e-6


def test_hex20_solid_cube_isotropic(dtc):
    """Affine fields are exact for both element types: C of a solid cube is the material's."""
    E, nu = 5600.0, 0.3
    gray = np.full((4, 4, 4), 14250, np.int16)
    with dtc.Solver(precision="fp64", rtol=1e-12, rotation_search=False) as s:
        r = s.solve([dtc.Domain(gray, elem_type=dtc.HEX20, E=E, nu=nu, delta=0.01)])[0]
    lam, mu = E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[range(3), range(3)] += 2 * mu
    C[3, 3] = C[4, 4] = C[5, 5] = mu
    assert rel(r["c"], C) < 1e-8


def test_mixed_element_types_rejected(dtc):
    gray = np.full((4, 4, 4), 100, np.int16)
    with dtc.Solver(precision="fp64", rtol=1e-8, rotation_search=False) as s:
        with pytest.raises(Exception, match="elem_type"):
            s.solve([dtc.Domain(gray), dtc.Domain(gray, elem_type=dtc.HEX20)])


# ---------------------------------------------------------------- multigrid inner preconditioner

def test_multigrid_cuts_inner_iterations(dtc, orc):
    """Same accuracy as block Jacobi with far fewer FP32 iterations (32^3, BV/TV 0.25)."""
    syn = dtc.synth
    gray = syn.bone_volume((32, 32, 32), 0.25, syn.seed_for(1, 3))
    dom = dtc.Domain(gray, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, E_voxel=syn.modulus_of_gray(gray))
    out = {}
    for pc in ("block", "mg"):
        with dtc.Solver(precision="mixed", rtol=1e-6, rotation_search=False, inner_precond=pc) as s:
            out[pc] = s.solve([dom])[0]
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False) as s:
        ref = s.solve([dom])[0]
    for pc in ("block", "mg"):
        assert out[pc]["status"] == 0
        assert rel(out[pc]["c"], ref["c"]) <= TOL_MIXED
    assert out["mg"]["iters"].max() * 4 < out["block"]["iters"].max()


def test_multigrid_uneven_sizes(dtc, orc):
    """Domains of different (also odd, non-cubic, tiny) sizes share one hierarchy build."""
    syn = dtc.synth
    pairs = [make_pair(dtc, orc, sh, 0.35, syn.seed_for(30, i), E_voxel=True)
             for i, sh in enumerate(((4, 4, 4), (5, 7, 6), (17, 9, 12), (16, 16, 16)))]
    refs = orc.solve_batch([p[1] for p in pairs])
    with dtc.Solver(precision="mixed", rtol=1e-10, rotation_search=False, inner_precond="mg") as s:
        res = s.solve([p[0] for p in pairs])
    for r, ref in zip(res, refs):
        assert r["status"] == 0
        assert rel(r["c"], ref["c"]) <= TOL_MIXED


@pytest.mark.parametrize("precision,precond,tol", [("fp64", "jacobi", 1e-7), ("mixed", "mg", 1e-5)])
def test_graph_replay_matches_direct_launches(dtc, batch, precision, precond, tol):
    """CG chunks replayed as CUDA graphs give the results of kernel-by-kernel launches (up to
    the order of the atomic dot-product sums)."""
    pairs, _ = batch
    out = {}
    for graphs in (True, False):
        with dtc.Solver(precision=precision, rtol=1e-8, rotation_search=False, inner_precond=precond,
                        graphs=graphs) as s:
            out[graphs] = s.solve([p[0] for p in pairs])
    for a, b in zip(out[True], out[False]):
        assert rel(a["c"], b["c"]) <= tol
        assert np.abs(a["iters"] - b["iters"]).max() <= 2


def test_hex20_multigrid_cuts_inner_iterations(dtc):
    """p-multigrid (HEX20 -> HEX08 of the same voxels -> halved grids) on a 16^3 HEX20 domain."""
    syn = dtc.synth
    gray = syn.bone_volume((16, 16, 16), 0.3, syn.seed_for(20, 30))
    dom = dtc.Domain(gray, elem_type=dtc.HEX20, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA,
                     E_voxel=syn.modulus_of_gray(gray))
    out = {}
    for pc in ("block", "mg"):
        with dtc.Solver(precision="mixed", rtol=1e-6, rotation_search=False, inner_precond=pc) as s:
            out[pc] = s.solve([dom])[0]
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False) as s:
        ref = s.solve([dom])[0]
    for pc in ("block", "mg"):
        assert out[pc]["status"] == 0
        assert rel(out[pc]["c"], ref["c"]) <= TOL_MIXED
    assert out["mg"]["iters"].max() * 4 < out["block"]["iters"].max()


@pytest.mark.parametrize("precond", ["mg", "jacobi"])
def test_hex20_tensor_core_matches_oracle(dtc, batch20, precond):
    """HEX20 FP32 element contraction on tcgen05 (3xTF32): same tolerance as the SIMT kernel."""
    pairs, refs = batch20
    with dtc.Solver(precision="mixed", rtol=1e-10, rotation_search=False, inner_precond=precond,
                    mixed_matvec="tensor") as s:
        res = s.solve([p[0] for p in pairs])
    for r, ref in zip(res, refs):
        assert r["status"] == 0
        assert rel(r["c"], ref["c"]) <= TOL_MIXED


@pytest.mark.parametrize("precond", ["block", "mg"])
def test_hex20_uniform_batch_matches_oracle(dtc, orc, precond):
    """A batch of HEX20 domains of one size (as c2): mixed path against the oracle."""
    pairs = [make_pair20(dtc, orc, (8, 8, 8), b, dtc.synth.seed_for(21, i), E_voxel=i == 2)
             for i, b in enumerate((0.2, 0.35, 0.5))]
    refs = orc.solve_batch([p[1] for p in pairs])
    with dtc.Solver(precision="mixed", rtol=1e-10, rotation_search=False, inner_precond=precond) as s:
        res = s.solve([p[0] for p in pairs])
    for r, ref in zip(res, refs):
        assert r["status"] == 0
        assert rel(r["c"], ref["c"]) <= TOL_MIXED
        assert rel(r["ff"], ref["ff"]) <= TOL_MIXED


@pytest.mark.parametrize("precision,precond,rtol", [("fp64", "block", 1e-10), ("mixed", "mg", 1e-8)])
def test_pipelined_passes_match_one_pass(dtc, precision, precond, rtol):
    """A batch of >= 256 domains is solved in 2 device passes, the host phase of the second
    overlapping the device work of the first; keep_displacements keeps one pass.  Same tensors, FP64
    iteration counts within 2, same statuses."""
    syn = dtc.synth
    rng = np.random.default_rng(17)
    doms = [dtc.Domain(syn.bone_volume((8, 8, 8), float(rng.uniform(0.15, 0.45)), syn.seed_for(12, i)),
                       E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, domain_number=i) for i in range(300)]
    doms[7] = dtc.Domain(np.zeros((8, 8, 8), np.int16), E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, domain_number=7)
    out = {}
    for keep in (False, True):
        with dtc.Solver(precision=precision, rtol=rtol, inner_precond=precond, rotation_search=True,
                        keep_displacements=keep, estimator="energy" if precision == "mixed" else "reaction") as s:
            out[keep] = s.solve(doms)
    for a, b in zip(out[False], out[True]):
        assert a["status"] == b["status"]
        assert (a["ne"], a["nn"], a["nb"], a["domain_number"]) == (b["ne"], b["nn"], b["nb"], b["domain_number"])
        if b["status"] == 0:
            assert rel(a["c"], b["c"]) <= (1e-9 if precision == "fp64" else 1e-6)
            if precision == "fp64":
                assert np.abs(a["iters"] - b["iters"]).max() <= 2   # atomic reduction order, as vs the oracle
    assert out[True][7]["status"] != 0


def test_autotuned_sweeps(dtc, batch):
    """mixed_matvec = auto: both sweep kernels are timed on the batch's tiles, the faster one
    solves; a second handle of the same size class reuses the cached decision (same timings)."""
    pairs, refs = batch
    doms = [p[0] for p in pairs]
    stats = []
    for _ in range(2):
        with dtc.Solver(precision="mixed", rtol=1e-10, rotation_search=False, inner_precond="mg",
                        mixed_matvec="auto") as s:
            res = s.solve(doms)
            stats.append(s.kernel_stats())
        for r, ref in zip(res, refs):
            assert r["status"] == 0
            assert rel(r["c"], ref["c"]) <= TOL_MIXED
    for st in stats:
        assert st["autotune_simt_sweep"]["launches"] == st["autotune_tc_sweep"]["launches"] == 3
        assert st["autotune_simt_sweep"]["ms_total"] > 0 and st["autotune_tc_sweep"]["ms_total"] > 0
    assert stats[0]["autotune_tc_sweep"]["ms_total"] == stats[1]["autotune_tc_sweep"]["ms_total"]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_device_passes_match_one_pass(dtc, batch, precision):
    """A batch cut into device passes (chunk_domains) gives the results of one pass: each later
    pass's voxel factors are uploaded through pinned memory on their own stream while the pass
    before solves, and the solve waits for that copy."""
    pairs, refs = batch
    doms = [p[0] for p in pairs]
    kw = dict(precision=precision, rtol=1e-10, rotation_search=False)
    if precision == "mixed":
        kw["inner_precond"] = "mg"
    with dtc.Solver(**kw) as s:
        one = s.solve(doms)
    with dtc.Solver(chunk_domains=2, **kw) as s:
        cut = s.solve(doms)
        again = s.solve(doms[::-1])[::-1]   # the slots alternate: a second batch reuses them
    for a, b, c, ref in zip(one, cut, again, refs):
        assert a["status"] == b["status"] == c["status"] == 0
        assert rel(b["c"], a["c"]) <= 1e-7 and rel(c["c"], a["c"]) <= 1e-7
        assert rel(b["c"], ref["c"]) <= (TOL_FP64 if precision == "fp64" else TOL_MIXED)
