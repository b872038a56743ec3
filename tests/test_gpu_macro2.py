"""Macro order 2 (20-node macro element, 60 load cases) on the GPU against the FP64 oracle,
through the C ABI: init_displ_hexe20 boundary modes (mod_write_deck.f90:118-279), projection
on phi_NN_hexe20 (mod_struct_calcmat.f90:254-280), the repaired quadratic load-case matrix
(:1780-2028) and the quadratic face sums (:368-401).

Tolerances as for macro order 1 (normwise relative against the oracle at rtol 1e-10):
FP64 path <= 1e-6, mixed path <= 1e-5; counts identical.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-6
TOL_MIXED = 1e-5


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pairs_for(dtc, orc, nen, shapes, seed0, E_voxel=False):
    syn = dtc.synth
    out = []
    for i, (shape, bvtv) in enumerate(shapes):
        gray = syn.bone_volume(shape, bvtv, syn.seed_for(seed0, i))
        ev = syn.modulus_of_gray(gray) if E_voxel else None
        d = dtc.Domain(gray, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, E_voxel=ev, elem_type=nen)
        o = orc.Domain(gray, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=1e-10, E_voxel=ev, nen=nen,
                       macro_order=2)
        out.append((d, o))
    return out


@pytest.fixture(scope="module")
def hex08(dtc, orc):
    pairs = pairs_for(dtc, orc, 8, [((10, 10, 10), 0.3), ((12, 12, 12), 0.45), ((9, 11, 10), 0.5)], 21)
    pairs += pairs_for(dtc, orc, 8, [((10, 10, 10), 0.35)], 22, E_voxel=True)
    return pairs, orc.solve_batch([p[1] for p in pairs])


@pytest.fixture(scope="module")
def hex20(dtc, orc):
    pairs = pairs_for(dtc, orc, 20, [((5, 5, 5), 0.5), ((6, 6, 6), 0.6)], 23)
    return pairs, orc.solve_batch([p[1] for p in pairs])


def check(res, refs, tol, fp64):
    for r, ref in zip(res, refs):
        assert r["status"] == ref["status"] == 0
        assert (r["ne"], r["nn"], r["nb"]) == (ref["ne"], ref["nn"], ref["nb"])
        assert r["ff"].shape == (60, 60) and r["kmacro"].shape == (60, 60) and r["iters"].shape == (60,)
        assert rel(r["c"], ref["c"]) <= tol
        assert rel(r["ff"], ref["ff"]) <= tol
        assert rel(r["kmacro"], ref["kmacro"]) <= tol
        if fp64:
            assert np.abs(r["iters"] - ref["iters"]).max() <= 2
        assert (r["iters"] > 0).all()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_hex08_macro_order2_matches_oracle(dtc, hex08, precision):
    pairs, refs = hex08
    kw = {"inner_precond": "mg"} if precision == "mixed" else {}
    with dtc.Solver(precision=precision, rtol=1e-10, rotation_search=True, macro_order=2, **kw) as s:
        res = s.solve([p[0] for p in pairs])
    check(res, refs, TOL_FP64 if precision == "fp64" else TOL_MIXED, precision == "fp64")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_macro_order2_energy_estimator_matches_oracle(dtc, hex08, precision):
    """ff from the 60 x 60 energy products u_a^T K u_b, whose blocks couple the three column
    passes (the solutions of the earlier passes stay on the device)."""
    pairs, refs = hex08
    kw = {"inner_precond": "mg"} if precision == "mixed" else {}
    with dtc.Solver(precision=precision, rtol=1e-10, rotation_search=False, macro_order=2, estimator="energy",
                    **kw) as s:
        res = s.solve([p[0] for p in pairs])
    check(res, refs, TOL_FP64 if precision == "fp64" else TOL_MIXED, precision == "fp64")


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_hex20_macro_order2_matches_oracle(dtc, hex20, precision):
    pairs, refs = hex20
    kw = {"inner_precond": "mg"} if precision == "mixed" else {}
    with dtc.Solver(precision=precision, rtol=1e-10, rotation_search=False, macro_order=2, **kw) as s:
        res = s.solve([p[0] for p in pairs])
    check(res, refs, TOL_FP64 if precision == "fp64" else TOL_MIXED, precision == "fp64")


def test_macro_order2_fields_match_oracle(dtc, orc):
    """The 60 displacement and reaction-force fields in the reference DOF numbering."""
    (d, o), = pairs_for(dtc, orc, 8, [((8, 8, 8), 0.4)], 24)
    ref = orc.solve_domain(o, with_arrays=True)
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=False, macro_order=2) as s:
        r, = s.solve([d], want_fields=True)
    assert r["displ"].shape == ref["displ"].shape == (60, 3 * ref["nn"])
    assert rel(r["displ"], ref["displ"]) <= TOL_FP64
    assert rel(r["force"], ref["force"]) <= TOL_FP64


def test_solid_cube_macro_order2_gives_isotropic_hooke(dtc):
    """TC01 isotropic, macro order 2 (regression/TC01-1_test_dev_dtc_isotropic-std-HEX08-ME2.meta)."""
    E, nu = 5600.0, 0.3
    lam, mu = E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[range(3), range(3)] += 2 * mu
    C[3, 3] = C[4, 4] = C[5, 5] = mu
    d = dtc.Domain(np.full((6, 6, 6), 14250, np.int16), E=E, nu=nu, delta=0.01)
    with dtc.Solver(precision="fp64", rtol=1e-12, rotation_search=False, macro_order=2) as s:
        r, = s.solve([d])
    assert r["status"] == 0
    assert rel(r["c"], C) < 1e-8


def test_macro_order2_needs_its_record(dtc):
    import ctypes as C
    d = dtc.Domain(np.full((4, 4, 4), 100, np.int16))
    with dtc.Solver(precision="fp64", macro_order=2) as s:
        ins = (dtc.capi.DomainIn * 1)(d.struct)
        outs = (dtc.capi.DomainOut * 1)()
        assert s.lib.dtc_solve_batch(s.handle, ins, 1, outs) == dtc.capi.DTC_ERR_INVALID_ARGUMENT
        assert b"macro2" in s.lib.dtc_last_error(s.handle)
        m2 = dtc.capi.Macro2Out()
        outs[0].macro2 = C.pointer(m2)
        assert s.lib.dtc_solve_batch(s.handle, ins, 1, outs) == dtc.capi.DTC_OK
        assert outs[0].status == 0 and m2.iters[59] > 0 and outs[0].iters[0] == 0
