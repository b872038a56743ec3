"""Known-answer tests of the FP64 oracle (the checker of the GPU path)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def hooke(E, nu):
    lam, mu = E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[range(3), range(3)] += 2 * mu
    C[3, 3] = C[4, 4] = C[5, 5] = mu
    return C


@pytest.mark.parametrize("macro_order", [1, 2])
@pytest.mark.parametrize("nen", [8, 20])
def test_solid_cube_gives_isotropic_hooke(orc, nen, macro_order):
    """TC01 isotropic (regression/TC01-1_test_dev_dtc_isotropic-std-HEX08-ME1.meta and -ME2): a
    fully solid domain; trilinear and serendipity elements reproduce the affine modes exactly,
    and the first six load cases of either macro element are those modes."""
    E, nu = 5600.0, 0.3
    r = orc.solve_domain(orc.Domain(np.full((4, 4, 4), 14250), E=E, nu=nu, delta=0.01, rtol=1e-13, nen=nen,
                                    macro_order=macro_order))
    assert r["status"] == 0
    assert r["ff"].shape == ((60, 60) if macro_order == 2 else (24, 24))
    C = hooke(E, nu)
    assert np.abs(r["c"] - C).max() / C.max() < 1e-9
    assert r["density"] == 1.0


@pytest.mark.parametrize("macro_order", [1, 2])
def test_kmacro_symmetric_and_rigid_modes(orc, macro_order):
    syn_phi = np.random.default_rng(4).random((6, 6, 6)) < 0.6
    r = orc.solve_domain(orc.Domain(syn_phi.astype(np.int32) * 20000, rtol=1e-12, macro_order=macro_order))
    K = r["kmacro"]
    nm = 20 if macro_order == 2 else 8
    assert K.shape == (3 * nm, 3 * nm)
    assert r["sym_k"] < 1e-6
    # translations of the macro element produce no force: dof index (k-1)*nm + l
    for c in range(3):
        t = np.zeros(3 * nm)
        t[c * nm:(c + 1) * nm] = 1.0
        assert np.abs(K @ t).max() < 1e-6 * np.abs(K).max()


def petsc_cg(A, b, dinv, rtol, max_it):
    """Independent Python restatement of PETSc 3.18 KSPSolve_CG + PCJACOBI +
    KSPConvergedDefault (preconditioned norm, zero guess)."""
    x = np.zeros_like(b)
    r = b.copy()
    z = dinv * r
    dp = np.linalg.norm(z)
    ttol = max(rtol * dp, 1e-50)
    if dp <= ttol:
        return x, 0
    beta = z @ r
    p = np.zeros_like(b)
    betaold = 1.0
    for i in range(max_it):
        p = z.copy() if i == 0 else z + (beta / betaold) * p
        w = A @ p
        dpi = p @ w
        betaold = beta
        a = beta / dpi
        x += a * p
        r -= a * w
        z = dinv * r
        dp = np.linalg.norm(z)
        if dp <= ttol:
            return x, i + 1
        beta = z @ r
    return x, max_it


def assemble(mesh, ke):
    nen = mesh["elems"].shape[1]
    nn = mesh["nn"]
    rows, cols, vals = [], [], []
    for el in mesh["elems"]:
        dofs = np.array([3 * (n - 1) + c for n in el for c in range(3)])
        keep = dofs >= 0
        rr, cc = np.meshgrid(dofs[keep], dofs[keep], indexing="ij")
        rows.append(rr.ravel()); cols.append(cc.ravel()); vals.append(ke[np.ix_(keep, keep)].ravel())
    return sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                         shape=(3 * nn, 3 * nn))


def test_petsc_cg_semantics_and_scipy_solution(orc):
    rng = np.random.default_rng(8)
    phi = (rng.random((5, 5, 5)) < 0.7).astype(np.int32) * 25000
    dom = orc.Domain(phi, rtol=1e-8, delta=0.05)
    r = orc.solve_domain(dom, with_arrays=True)
    mesh = orc.mesh_domain(dom)
    ke = orc.element_stiffness(8, 5600.0, 5 * 0.05 * 0.05, 0.3)
    A = assemble(mesh, ke)
    n = A.shape[0]
    bc = np.zeros(n, bool)
    for b in mesh["bnode_ids"]:
        bc[3 * (b - 1): 3 * b] = True
    free = ~bc
    Aff = A[free][:, free]
    dinv = 1.0 / Aff.diagonal()
    for lc in (0, 5, 23):
        g = np.zeros(n)
        g[bc] = mesh["bnode_vals"][lc].reshape(-1, 3).ravel()[: bc.sum()] if False else 0.0
        # prescribed values in dof order
        vals = mesh["bnode_vals"][lc]
        for k, b in enumerate(mesh["bnode_ids"]):
            g[3 * (b - 1): 3 * b] = vals[3 * k: 3 * k + 3]
        b_f = -(A @ g)[free]
        x, its = petsc_cg(Aff, b_f, dinv, 1e-8, 100000)
        assert abs(its - r["iters"][lc]) <= 1
        u_ref = spla.spsolve(Aff.tocsc(), b_f)
        u = r["displ"][lc][free]
        assert np.abs(u - u_ref).max() <= 1e-6 * np.abs(u_ref).max()
        # reactions AA_org * u with the prescribed values inserted (mod_dtc_main_subroutines.f90:1092-1123)
        full = g.copy()
        full[free] = u
        assert np.abs(A @ full - r["force"][lc]).max() <= 1e-9 * np.abs(r["force"][lc]).max()


def random_rotation(rng):
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def mandel_rotation(aa):
    s2 = np.sqrt(2.0)
    B = np.zeros((6, 6))
    pairs = [(0, 1), (0, 2), (1, 2)]
    for col in range(3):
        a = aa[:, col]
        B[:, col] = [a[0] ** 2, a[1] ** 2, a[2] ** 2, s2 * a[1] * a[0], s2 * a[0] * a[2], s2 * a[1] * a[2]]
    for q, (i, j) in enumerate(pairs):
        ai, aj = aa[:, i], aa[:, j]
        B[:, 3 + q] = [s2 * ai[0] * aj[0], s2 * ai[1] * aj[1], s2 * ai[2] * aj[2],
                       ai[1] * aj[0] + aj[1] * ai[0], ai[0] * aj[2] + aj[0] * ai[2], ai[1] * aj[2] + aj[1] * ai[2]]
    return B


@pytest.mark.slow
def test_rotation_search_recovers_orthotropic_axes(orc):
    """CR2 of a rotated orthotropic tensor returns to (near) zero off-diagonal energy and a
    diagonal ordered E11 <= E22 <= E33 after the permutation fix-up."""
    rng = np.random.default_rng(2)
    E0 = np.diag([9000.0, 12000.0, 15000.0, 3000.0, 4000.0, 5000.0])
    E0[0, 1] = E0[1, 0] = 3000.0
    E0[0, 2] = E0[2, 0] = 3500.0
    E0[1, 2] = E0[2, 1] = 4000.0
    B = mandel_rotation(random_rotation(rng))
    ee = B.T @ E0 @ B
    r = orc.rotation_search(ee)
    assert r["cr2"]["crit"] < 1e-6 * np.abs(ee).max() ** 2
    d = np.diag(r["cr2"]["ee"])
    assert d[0] <= d[1] <= d[2]
    assert np.allclose(sorted(d[:3]), [9000, 12000, 15000], rtol=1e-5)
