"""dtc_rotation_search_noalloc: the rotation search for callers that cannot allocate device
memory when they call it (for example while capturing a CUDA stream, or when every device
buffer must come from the host application's own pool).  The entry point keeps its scratch in
a fixed device array; these tests check, through the C ABI, that two calls in a row give the
results of the regular path (dtc_solve_batch with rotation_search = 1) and the oracle's argmin
indices, on the default stream and on a non-blocking stream, also when the non-blocking call
is the first use of the library in a fresh process.

The file name makes pytest collect it last."""
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def _domains(dtc):
    syn = dtc.synth
    return [dtc.Domain(syn.bone_volume((10, 10, 10), b, syn.seed_for(8, i)), E=syn.E_CONST, nu=syn.NU,
                       delta=syn.DELTA) for i, b in enumerate((0.35, 0.5, 0.6))]


def _call(dtc, ee_d, n, stream_ptr):
    import torch
    dev = ee_d.device
    ang = torch.full((n, 2, 3), -7, dtype=torch.int64, device=dev)
    jj = torch.zeros((n, 2), dtype=torch.int32, device=dev)
    crit = torch.full((n, 2), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    rc = dtc.capi.load().dtc_rotation_search_noalloc(ee_d.data_ptr(), n, ang.data_ptr(), jj.data_ptr(),
                                                     crit.data_ptr(), stream_ptr)
    assert rc == dtc.capi.DTC_OK
    torch.cuda.synchronize()
    return ang.cpu().numpy(), jj.cpu().numpy(), crit.cpu().numpy()


@pytest.mark.parametrize("stream", ["default", "nonblocking"])
def test_noalloc_rotation_matches_solve_batch(dtc, orc, stream):
    import torch

    doms = _domains(dtc)
    with dtc.Solver(precision="fp64", rtol=1e-10, rotation_search=True) as s:
        ref = s.solve(doms)
    n = len(doms)
    ee = np.stack([r["ee"].reshape(-1, order="F") for r in ref])   # column-major 6x6 per domain
    orc_ref = [orc.rotation_search(r["ee"]) for r in ref]
    dev = torch.device("cuda", 0)
    ee_d = torch.tensor(ee, dtype=torch.float64, device=dev)
    st = torch.cuda.Stream(device=dev) if stream == "nonblocking" else None
    for _ in range(2):   # the shared scratch keeps the previous call's contents
        if st is not None:
            with torch.cuda.stream(st):
                a, j, c = _call(dtc, ee_d, n, st.cuda_stream)
        else:
            a, j, c = _call(dtc, ee_d, n, None)
        for i, r in enumerate(ref):
            for w, k in enumerate(("cr1", "cr2")):
                assert j[i, w] == r[k]["iters"] == orc_ref[i][k]["iters"]
                assert c[i, w] == r[k]["crit"] == orc_ref[i][k]["crit"]
                assert (a[i, w] == orc_ref[i][k]["ang"]).all()
            # CR1 records the angle the search found: ang * pi / (180 (10^jj - 1))
            alpha = a[i, 0, 0] * np.pi / (180.0 * (10.0 ** j[i, 0] - 1.0))
            assert alpha == pytest.approx(r["cr1"]["angle"], rel=1e-12, abs=1e-15)
    too_many = 1025
    z = torch.zeros(too_many * 6, dtype=torch.int64, device=dev)
    assert dtc.capi.load().dtc_rotation_search_noalloc(ee_d.data_ptr(), too_many, z.data_ptr(), z.data_ptr(),
                                                       z.data_ptr(), None) == dtc.capi.DTC_ERR_INVALID_ARGUMENT


FRESH = textwrap.dedent("""
    import sys
    import numpy as np
    import torch
    sys.path.insert(0, {root!r})
    import __graft_entry__ as ge
    dtc = ge.load_package()
    lib = dtc.capi.load()
    dev = torch.device("cuda", 0)
    iso = np.zeros((6, 6)); iso[:3, :3] = 5000.0; iso[range(3), range(3)] += 6000.0
    iso[range(3, 6), range(3, 6)] = 1500.0
    ee = torch.tensor(iso.reshape(1, 36), dtype=torch.float64, device=dev)
    st = torch.cuda.Stream(device=dev)
    out = []
    for _ in range(2):
        ang = torch.zeros((1, 2, 3), dtype=torch.int64, device=dev)
        jj = torch.zeros((1, 2), dtype=torch.int32, device=dev)
        crit = torch.zeros((1, 2), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        with torch.cuda.stream(st):
            rc = lib.dtc_rotation_search_noalloc(ee.data_ptr(), 1, ang.data_ptr(), jj.data_ptr(), crit.data_ptr(),
                                                 st.cuda_stream)
        assert rc == 0, rc
        st.synchronize()
        out.append((ang.cpu().numpy().tolist(), jj.cpu().numpy().tolist(), crit.cpu().numpy().tolist()))
    print(repr(out))
""")


def test_noalloc_first_call_on_nonblocking_stream_in_fresh_process(dtc, orc):
    """The first call on a device uploads the sweep tables; work on a non-blocking stream must
    see them (the upload is complete before the call returns)."""
    p = subprocess.run([sys.executable, "-c", FRESH.format(root=str(ROOT))], capture_output=True, text=True,
                       timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr
    out = eval(p.stdout.strip().splitlines()[-1])
    iso = np.zeros((6, 6))
    iso[:3, :3] = 5000.0
    iso[range(3), range(3)] += 6000.0
    iso[range(3, 6), range(3, 6)] = 1500.0
    ref = orc.rotation_search(iso)
    for ang, jj, crit in out:
        for w, k in enumerate(("cr1", "cr2")):
            assert ang[0][w] == list(ref[k]["ang"])
            assert jj[0][w] == ref[k]["iters"]
            assert crit[0][w] == ref[k]["crit"]
