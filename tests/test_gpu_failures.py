"""Per-domain failure statuses and the tensor-core kernels' error path, on the device.

Failures are made on the host side (bad moduli in the input, a shortened wait limit); nothing
here faults or hangs the GPU.  A failing domain must not disturb the other domains of its
batch, and the handle (and the CUDA context) must stay usable.
  * a NaN modulus             -> DTC_DOMAIN_NONFINITE (PETSc: KSP_DIVERGED_NANORINF)
  * moduli of mixed sign       -> DTC_DOMAIN_BREAKDOWN (KSP_DIVERGED_INDEFINITE_PC / _MAT)
    (an all-negative domain is NOT a breakdown: CG on -K with the -D^-1 preconditioner has
    the iterates of K, which the oracle's restatement of KSPSolve_CG reproduces)
  * a tensor-core wait that runs out -> dtc_solve_batch returns DTC_ERR_INTERNAL
Reference skip semantics: f-src/mod_dtc_main_subroutines.f90:276-277,
f-src_main/struct_process.f90:1385 (a failed domain is skipped, the loop goes on).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def domains(dtc, kinds):
    syn = dtc.synth
    g = syn.bone_volume((8, 8, 8), 0.5, syn.seed_for(9, 50))
    out = []
    for kind in kinds:
        E = syn.modulus_of_gray(g).copy()
        if kind == "nan":
            E[tuple(np.argwhere(E > 0)[0])] = np.nan
        elif kind == "half":
            E[:, :, :4] *= -1
        elif kind == "one":
            bone = np.argwhere(E > 0)
            E[tuple(bone[len(bone) // 2])] *= -50
        elif kind == "allneg":
            E = -E
        out.append((g, E))
    return out


def solve(dtc, pairs, **kw):
    syn = dtc.synth
    doms = [dtc.Domain(g, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, E_voxel=E, domain_number=i)
            for i, (g, E) in enumerate(pairs)]
    with dtc.Solver(rotation_search=False, **kw) as s:
        return s.solve(doms)


@pytest.mark.parametrize("kw", [dict(precision="fp64", rtol=1e-10),
                                dict(precision="mixed", rtol=1e-8, inner_precond="mg", estimator="energy"),
                                dict(precision="mixed", rtol=1e-8, inner_precond="jacobi")])
def test_bad_moduli_statuses(dtc, orc, kw):
    kinds = ["ok", "nan", "half", "one", "allneg", "ok"]
    pairs = domains(dtc, kinds)
    res = solve(dtc, pairs, **kw)
    healthy = solve(dtc, [pairs[0]], **kw)[0]
    syn = dtc.synth
    for kind, (g, E), r in zip(kinds, pairs, res):
        ref = orc.solve_domain(orc.Domain(g, E=syn.E_CONST, nu=syn.NU, delta=syn.DELTA, rtol=1e-10, E_voxel=E))
        if kind == "ok":
            assert r["status"] == dtc.DOMAIN_OK
            # the failing neighbours of the batch do not change a healthy domain's result (up to
            # the summation order of the dot products, which follows the batch's CTA schedule)
            tol = 1e-9 if kw["precision"] == "fp64" else 1e-6
            assert np.abs(r["c"] - healthy["c"]).max() <= tol * np.abs(healthy["c"]).max()
        elif kind == "nan":
            assert r["status"] == ref["status"] == dtc.DOMAIN_NONFINITE
        elif kind in ("half", "one"):
            assert ref["status"] == dtc.DOMAIN_BREAKDOWN
            if kw["precision"] == "fp64":
                assert r["status"] == dtc.DOMAIN_BREAKDOWN
            else:   # the FP32 inner solve may see the sign change first as a non-finite step
                assert r["status"] in (dtc.DOMAIN_BREAKDOWN, dtc.DOMAIN_NONFINITE, dtc.DOMAIN_MAX_IT)
        elif kind == "allneg":
            assert ref["status"] == dtc.DOMAIN_OK
            if kw["precision"] == "fp64":
                assert r["status"] == dtc.DOMAIN_OK
                assert np.abs(r["c"] - ref["c"]).max() <= 1e-6 * np.abs(ref["c"]).max()


def test_tensor_core_wait_timeout_is_reported(dtc):
    """Per-round completion waits allowed no poll give up: the call returns DTC_ERR_INTERNAL
    (not a fault; the kernel still drains its MMAs with the full bound before freeing tensor
    memory), and the device stays usable for the next handle."""
    pairs = domains(dtc, ["ok", "ok"])
    with pytest.raises(dtc.DTCError) as ei:
        solve(dtc, pairs, precision="mixed", rtol=1e-8, inner_precond="block", mixed_matvec="tensor",
              tc_wait_spins=-1)
    assert ei.value.code == dtc.capi.DTC_ERR_INTERNAL
    ok = solve(dtc, pairs, precision="mixed", rtol=1e-8, inner_precond="block", mixed_matvec="tensor")
    ref = solve(dtc, pairs, precision="fp64", rtol=1e-10)
    for r, f in zip(ok, ref):
        assert r["status"] == dtc.DOMAIN_OK
        assert np.abs(r["c"] - f["c"]).max() <= 1e-5 * np.abs(f["c"]).max()
