"""Adjoint dL/dE_voxel (dtc_energy_grad) against an FP64 reference gradient built from the
oracle's displacements, against central finite differences, through torch.autograd, and
across memory chunks whose displacements are checkpointed to the host."""
import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

MEPS = np.array([1e6, 1e6, 1e6, -1e6, -1e6, 1e6])


def dloss_dff(dc, L, delta):
    """dL/dff through C = fv * meps; fv = face sums of ff rows / face areas
    (f-src/mod_struct_calcmat.f90:345-359, 434-439).  dc, result: [row, col] arrays."""
    X, Y, Z = (L[0] * delta, L[1] * delta, L[2] * delta)
    rows = [([2, 3, 6, 7], 1 / (Y * Z)), ([11, 12, 15, 16], 1 / (X * Z)), ([21, 22, 23, 24], 1 / (X * Y))]
    shear = [([3, 4, 7, 8], 0.5 / (X * Z), [10, 11, 14, 15], 0.5 / (Y * Z)),
             ([5, 6, 7, 8], 0.5 / (X * Y), [18, 19, 22, 23], 0.5 / (Y * Z)),
             ([13, 14, 15, 16], 0.5 / (X * Y), [19, 20, 23, 24], 0.5 / (X * Z))]
    lff = np.zeros((24, 24))
    for c in range(6):
        g = dc[:, c] * MEPS[c]
        for i, (rr, w) in enumerate(rows):
            for r in rr:
                lff[r - 1, c] += g[i] * w
        for i, (r1, w1, r2, w2) in enumerate(shear):
            for r in r1:
                lff[r - 1, c] += g[3 + i] * w1
            for r in r2:
                lff[r - 1, c] += g[3 + i] * w2
    return lff


def reference_gradient(orc, dtc, gray, ev, dc, delta, nu):
    """FP64: dL/dE_v = a * sum_ab G_ab u_a,v^T Khat u_b,v, G = vv^-1 dL/dff (oracle solve)."""
    o = orc.Domain(gray, E=5600.0, nu=nu, delta=delta, rtol=1e-12, E_voxel=ev)
    r = orc.solve_domain(o, with_arrays=True)
    L = gray.shape[::-1]
    vv = np.load(GOLDEN / "vv_lin_eps1e-6.npy")
    G = np.linalg.inv(vv) @ dloss_dff(dc, L, delta)
    kh = dtc.element_stiffness(8, 1.0, 1.0, nu)
    a = L[0] * delta * delta
    g = np.zeros(gray.size)
    dofs = (3 * (r["elems"][:, :, None] - 1) + np.arange(3)).reshape(len(r["elems"]), 24)
    U = r["displ"].T[dofs]                         # (ne, 24 dofs, 24 load cases)
    KU = np.einsum("ij,ejb->eib", kh, U)
    g[r["elem_voxel"]] = a * np.einsum("eia,ab,eib->e", U, G, KU)
    return g.reshape(gray.shape), r["c"]


def loss_and_dc(C, target):
    return float(((C - target) ** 2).sum()), 2.0 * (C - target)


@pytest.fixture(scope="module")
def case(dtc):
    syn = dtc.synth
    gray = syn.bone_volume((10, 10, 10), 0.35, syn.seed_for(4, 1))
    ev = syn.modulus_of_gray(gray)
    rng = np.random.default_rng(5)
    target = np.diag(rng.uniform(3000, 15000, 6))
    return gray, ev, target


def grad_of(dtc, gray, ev, target, **kw):
    with dtc.Solver(rotation_search=False, keep_displacements=True, **kw) as s:
        r = s.solve([dtc.Domain(gray, E=5600.0, nu=dtc.synth.NU, delta=dtc.synth.DELTA, E_voxel=ev)])[0]
        L, dc = loss_and_dc(r["c"], target)
        g = [np.zeros(gray.shape, np.float32)]
        s.energy_grad(dc[None], g)
    return g[0], r["c"], L


def test_adjoint_matches_fp64_reference_gradient(dtc, orc, case):
    gray, ev, target = case
    g, C, _ = grad_of(dtc, gray, ev, target, precision="fp64", rtol=1e-12)
    _, dc = loss_and_dc(C, target)
    gref, Cref = reference_gradient(orc, dtc, gray, ev, dc, dtc.synth.DELTA, dtc.synth.NU)
    assert np.abs(C - Cref).max() <= 1e-8 * np.abs(Cref).max()
    assert np.abs(g - gref).max() <= 1e-5 * np.abs(gref).max()
    assert np.all(g[gray < 1] == 0)


def test_adjoint_central_differences(dtc, case):
    """32 random kept voxels, h = 1e-3 E_v, FP64 solves at rtol 1e-12."""
    gray, ev, target = case
    g, C, _ = grad_of(dtc, gray, ev, target, precision="fp64", rtol=1e-12)
    rng = np.random.default_rng(11)
    kept = np.flatnonzero(g.ravel() != 0)
    pick = rng.choice(kept, size=min(32, kept.size), replace=False)
    doms = []
    for v in pick:
        for sgn in (1, -1):
            e = ev.copy().ravel()
            e[v] *= 1 + sgn * 1e-3
            doms.append(dtc.Domain(gray, E=5600.0, nu=dtc.synth.NU, delta=dtc.synth.DELTA,
                                   E_voxel=e.reshape(ev.shape)))
    with dtc.Solver(precision="fp64", rtol=1e-12, rotation_search=False) as s:
        res = s.solve(doms)
    for k, v in enumerate(pick):
        lp = loss_and_dc(res[2 * k]["c"], target)[0]
        lm = loss_and_dc(res[2 * k + 1]["c"], target)[0]
        fd = (lp - lm) / (2e-3 * ev.ravel()[v])
        assert abs(fd - g.ravel()[v]) <= 2e-3 * np.abs(g).max(), (v, fd, g.ravel()[v])


def test_mixed_adjoint_close_to_fp64(dtc, case):
    gray, ev, target = case
    g64, _, _ = grad_of(dtc, gray, ev, target, precision="fp64", rtol=1e-12)
    gmx, _, _ = grad_of(dtc, gray, ev, target, precision="mixed", rtol=1e-7, inner_precond="mg", estimator="energy")
    assert np.abs(gmx - g64).max() <= 1e-3 * np.abs(g64).max()


def test_adjoint_checkpointed_chunks(dtc):
    """A batch solved in 3 device passes (2 checkpointed to the host) gives the same gradients."""
    syn = dtc.synth
    grays = [syn.bone_volume((8, 8, 8), 0.4, syn.seed_for(4, 10 + i)) for i in range(5)]
    doms = [dtc.Domain(g, E=5600.0, nu=syn.NU, delta=syn.DELTA, E_voxel=syn.modulus_of_gray(g)) for g in grays]
    dc = np.random.default_rng(3).standard_normal((5, 6, 6))
    out = {}
    for chunk in (0, 2):
        with dtc.Solver(precision="fp64", rtol=1e-12, rotation_search=False, keep_displacements=True,
                        chunk_domains=chunk) as s:
            s.solve(doms)
            g = [np.zeros(gr.shape, np.float32) for gr in grays]
            s.energy_grad(dc, g)
        out[chunk] = np.stack(g)
    assert np.abs(out[0]).max() > 0
    assert np.abs(out[2] - out[0]).max() <= 1e-6 * np.abs(out[0]).max()


def test_autograd_function(dtc):
    torch = pytest.importorskip("torch")
    from importlib import import_module
    ag = import_module(dtc.__name__ + ".autograd")
    syn = dtc.synth
    grays = [syn.bone_volume((8, 8, 8), 0.4, syn.seed_for(4, 20 + i)) for i in range(2)]
    E = torch.tensor(np.stack([syn.modulus_of_gray(g) for g in grays]), requires_grad=True)
    model = ag.EffectiveStiffness(grays, precision="fp64", rtol=1e-12)
    target = torch.eye(6, dtype=torch.float64) * 5000.0
    C = model(E)
    loss = ((C - target) ** 2).sum()
    loss.backward()
    # the same gradient straight from the C ABI
    dc = (2.0 * (C.detach() - target)).numpy()
    g = [np.zeros(gr.shape, np.float32) for gr in grays]
    model.solver.energy_grad(dc, g)
    assert torch.allclose(E.grad, torch.from_numpy(np.stack(g)))
    assert float(E.grad.abs().max()) > 0
    model.close()


def test_autograd_function_device_tensors(dtc):
    """E as a CUDA tensor: moduli in and gradient out through the device-pointer entries
    (dtc_solve_batch_device_moduli, dtc_energy_grad_device); same C and gradient as the host path."""
    torch = pytest.importorskip("torch")
    from importlib import import_module
    ag = import_module(dtc.__name__ + ".autograd")
    syn = dtc.synth
    grays = [syn.bone_volume((8, 8, 8), 0.4, syn.seed_for(4, 30 + i)) for i in range(3)]
    E0 = np.stack([syn.modulus_of_gray(g) for g in grays])
    target = torch.eye(6, dtype=torch.float64) * 5000.0
    out = {}
    for where in ("cpu", "cuda"):
        E = torch.tensor(E0, requires_grad=True, device=where)
        model = ag.EffectiveStiffness(grays, precision="fp64", rtol=1e-12)
        C = model(E)
        assert C.device.type == where
        loss = ((C - target.to(where)) ** 2).sum()
        loss.backward()
        assert E.grad.device.type == where
        out[where] = (C.detach().cpu().numpy(), E.grad.detach().cpu().numpy())
        model.close()
    assert np.abs(out["cuda"][0] - out["cpu"][0]).max() <= 1e-9 * np.abs(out["cpu"][0]).max()
    assert np.abs(out["cuda"][1] - out["cpu"][1]).max() <= 1e-6 * np.abs(out["cpu"][1]).max()
    assert np.abs(out["cuda"][1]).max() > 0
