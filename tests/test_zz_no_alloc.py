"""dtc_rotation_search_noalloc: the rotation search for callers that cannot allocate device
memory when they call it (for example while capturing a CUDA stream, or when every device
buffer must come from the host application's own pool).  The entry point keeps its scratch in
a fixed device array; this test checks, through the C ABI, that two calls in a row give the
results of the regular path (dtc_solve_batch with rotation_search = 1).

The file name makes pytest collect it last."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_rotation_matches_solve_batch(dtc):
    import torch

    syn = dtc.synth
    doms = [dtc.Domain(syn.bone_volume((10, 10, 10), b, syn.seed_for(8, i)), E=syn.E_CONST, nu=syn.NU,
                       delta=syn.DELTA) for i, b in enumerate((0.35, 0.5, 0.6))]
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=True) as s:
        ref = s.solve(doms)
    n = len(doms)
    ee = np.stack([r["ee"].reshape(-1, order="F") for r in ref])   # column-major 6x6 per domain
    lib = dtc.capi.load()
    dev = torch.device("cuda", 0)
    ee_d = torch.tensor(ee, dtype=torch.float64, device=dev)
    for _ in range(2):   # the shared scratch keeps the previous call's contents
        ang = torch.full((n, 2, 3), -7, dtype=torch.int64, device=dev)
        jj = torch.zeros((n, 2), dtype=torch.int32, device=dev)
        crit = torch.full((n, 2), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = lib.dtc_rotation_search_noalloc(ee_d.data_ptr(), n, ang.data_ptr(), jj.data_ptr(), crit.data_ptr(),
                                             None)
        assert rc == dtc.capi.DTC_OK
        torch.cuda.synchronize()
        a, j, c = ang.cpu().numpy(), jj.cpu().numpy(), crit.cpu().numpy()
        for i, r in enumerate(ref):
            for w, k in enumerate(("cr1", "cr2")):
                assert j[i, w] == r[k]["iters"]
                assert abs(c[i, w] - r[k]["crit"]) <= 1e-9 + 1e-6 * abs(r[k]["crit"])
            # CR1 records the angle the search found: ang * pi / (180 (10^jj - 1))
            alpha = a[i, 0, 0] * np.pi / (180.0 * (10.0 ** j[i, 0] - 1.0))
            assert alpha == pytest.approx(r["cr1"]["angle"], rel=1e-12, abs=1e-15)
    too_many = 1025
    assert lib.dtc_rotation_search_noalloc(ee_d.data_ptr(), too_many, ang.data_ptr(), jj.data_ptr(),
                                           crit.data_ptr(), None) == dtc.capi.DTC_ERR_INVALID_ARGUMENT
