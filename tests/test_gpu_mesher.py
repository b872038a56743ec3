"""The device mesher (dtc_mesh_batch; dtc_options.device_mesher in dtc_solve_batch) against the
host planner (dtc_mesh_domain), which tests/test_mesher.py pins bit for bit to the oracle's
literal restatement of gen_quadmesh_from_phi / generate_boundaries
(f-src/mod_gen_quadmesh.f90:22-679, f-src/mod_struct_preprocess.f90:490-738): statuses,
counts, element connectivity in reference node ids, node coordinates, constrained-node ids and
their prescribed values must be identical."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def same(a, b):
    assert a["status"] == b["status"]
    assert (a["ne"], a["nn"], a["nb"]) == (b["ne"], b["nn"], b["nb"])
    assert a["last_elem_partial"] == b["last_elem_partial"]
    for k in ("elems", "nodes", "bnode_ids", "bnode_vals"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("nen", [8, 20])
def test_device_mesher_random_volumes(dtc, nen):
    rng = np.random.default_rng(101 + nen)
    doms = []
    for _ in range(150 if nen == 8 else 60):
        L = rng.integers(1, 10, size=3)
        p = rng.random() * 0.7
        phi = (rng.random((L[2], L[1], L[0])) < p).astype(np.int16) * int(rng.integers(1, 30000))
        doms.append(dtc.Domain(phi, elem_type=nen, delta=0.05, xa_n=tuple(int(v) for v in rng.integers(1, 40, 3))))
    with dtc.Solver() as s:
        dev = s.mesh_batch(doms)
    for d, m in zip(doms, dev):
        same(m, dtc.mesh_domain(d))


def test_device_mesher_benchmark_domains(dtc):
    """Domains drawn like the headline batch (32^3) and the uneven one (16-64 voxels per edge)."""
    syn = dtc.synth
    rng = np.random.default_rng(7)
    doms = [dtc.Domain(syn.bone_volume((32, 32, 32), float(b), syn.seed_for(1, 500 + i)))
            for i, b in enumerate(rng.uniform(0.1, 0.4, 6))]
    doms += [dtc.Domain(syn.bone_volume((int(L),) * 3, float(b), syn.seed_for(3, 500 + i)))
             for i, (L, b) in enumerate(zip((16, 24, 48, 64), (0.05, 0.45, 0.2, 0.3)))]
    with dtc.Solver() as s:
        dev = s.mesh_batch(doms)
    for d, m in zip(doms, dev):
        same(m, dtc.mesh_domain(d))


@pytest.mark.parametrize("dtype", [np.int8, np.int16, np.int32])
def test_device_mesher_gray_types(dtc, dtype):
    rng = np.random.default_rng(3)
    phi = rng.integers(-100, 100, size=(6, 7, 5)).astype(dtype)
    d = dtc.Domain(phi, llimit=20)
    with dtc.Solver() as s:
        same(s.mesh_batch([d])[0], dtc.mesh_domain(d))


def test_solve_with_device_mesher(dtc):
    """dtc_solve_batch with the device mesher gives the host-mesher results (and fields in the
    same reference numbering)."""
    syn = dtc.synth
    doms = [dtc.Domain(syn.bone_volume((10, 10, 10), b, syn.seed_for(8, 60 + i)), E=syn.E_CONST, nu=syn.NU,
                       delta=syn.DELTA) for i, b in enumerate((0.3, 0.5, 0.02))]
    out = {}
    for dm in (False, True):
        with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False, device_mesher=dm) as s:
            out[dm] = s.solve(doms, want_fields=True)
    for a, b in zip(out[True], out[False]):
        assert a["status"] == b["status"]
        assert (a["ne"], a["nn"], a["nb"]) == (b["ne"], b["nn"], b["nb"])
        if a["status"] == 0:
            assert np.abs(a["c"] - b["c"]).max() <= 1e-9 * np.abs(b["c"]).max()
            assert np.abs(a["displ"] - b["displ"]).max() <= 1e-9 * np.abs(b["displ"]).max()


@pytest.mark.parametrize("nen", [8, 20])
def test_device_mesher_macro_order2(dtc, nen):
    """The 60 prescribed values per constrained DOF of macro order 2, from the device mesher's
    plans, equal the host planner's (tests/test_mesher.py pins those to the oracle); and a solve
    with the device mesher gives the host-mesher solve's 60 x 60 leaves."""
    rng = np.random.default_rng(211 + nen)
    doms = []
    for _ in range(20):
        L = rng.integers(2, 9, size=3)
        phi = (rng.random((L[2], L[1], L[0])) < 0.6).astype(np.int16) * 1000
        doms.append(dtc.Domain(phi, elem_type=nen, delta=0.05, xa_n=tuple(int(v) for v in rng.integers(1, 40, 3))))
    with dtc.Solver() as s:
        dev = s.mesh_batch(doms, macro_order=2)
    for d, m in zip(doms, dev):
        ref = dtc.mesh_domain(d, macro_order=2)
        same(m, ref)
        assert m["bnode_vals"].shape == (60, 3 * m["nb"])
    syn = dtc.synth
    sd = [dtc.Domain(syn.bone_volume((8, 8, 8), b, syn.seed_for(8, 90 + i)), elem_type=nen, E=syn.E_CONST, nu=syn.NU,
                     delta=syn.DELTA) for i, b in enumerate((0.35, 0.5))]
    out = {}
    for dm in (False, True):
        with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False, device_mesher=dm, macro_order=2) as s:
            out[dm] = s.solve(sd)
    for a, b in zip(out[True], out[False]):
        assert a["status"] == b["status"] == 0
        assert np.abs(a["kmacro"] - b["kmacro"]).max() <= 1e-9 * np.abs(b["kmacro"]).max()
