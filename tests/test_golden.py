"""Pins of the oracle and of the library's host FE code against the reference's own tables
(tests/golden/, generated by tests/golden/make_golden.py from the reference source)."""
import json

import numpy as np
import pytest

from conftest import GOLDEN


def table_factor(nen, E, a, nu):
    if nen == 8:   # mod_linfe.f90:182
        return E * a / (144.0 * (2.0 * nu ** 2 + nu - 1.0))
    return E * a * (nu * 2.0) / (256.0 * (2.0 * nu ** 2 + nu - 1.0) * 2.0 * nu)  # :904


@pytest.mark.parametrize("nen,name", [(8, "ke08"), (20, "ke20")])
@pytest.mark.parametrize("nu", [0.3, 0.25])
def test_oracle_element_stiffness_equals_reference_table(orc, nen, name, nu):
    E, a = 5600.0, 0.5 * 0.01
    ref = np.load(GOLDEN / f"{name}_table_nu{nu}.npy") * table_factor(nen, E, a, nu)
    ke = orc.element_stiffness(nen, E, a, nu)
    assert np.abs(ke - ref).max() / np.abs(ref).max() < 1e-13


@pytest.mark.parametrize("nen,name", [(8, "ke08"), (20, "ke20")])
@pytest.mark.parametrize("nu", [0.3, 0.25])
def test_library_element_stiffness_equals_reference_table(dtc, nen, name, nu):
    E, a = 7000.0, 1.6 * 0.05
    ref = np.load(GOLDEN / f"{name}_table_nu{nu}.npy") * table_factor(nen, E, a, nu)
    ke = dtc.element_stiffness(nen, E, a, nu)
    assert np.abs(ke - ref).max() / np.abs(ref).max() < 1e-13
    assert np.abs(ke - ke.T).max() <= 1e-12 * np.abs(ke).max()
    # rigid-body translations are in the null space
    for c in range(3):
        t = np.zeros(3 * nen)
        t[c::3] = 1.0
        assert np.abs(ke @ t).max() < 1e-10 * np.abs(ke).max()


def test_boundary_modes_and_loadcase_matrix(orc):
    uu = orc.boundary_modes(1e-6)
    vv = orc.loadcase_matrix(1e-6)
    assert np.array_equal(uu, np.load(GOLDEN / "uu_hexe8_eps1e-6.npy"))
    assert np.array_equal(vv, np.load(GOLDEN / "vv_lin_eps1e-6.npy"))
    # vv is the component-major flattening of uu (mod_struct_calcmat.f90:1684-1770 vs
    # mod_write_deck.f90:63-116)
    flat = np.zeros((24, 24))
    for k in range(3):
        for l in range(8):
            flat[k * 8 + l] = uu[l, k]
    assert np.array_equal(vv, flat)
    assert abs(np.linalg.cond(vv) - 21.6464) < 1e-3


def test_golden_meta_records_sources():
    meta = json.loads((GOLDEN / "golden_meta.json").read_text())
    assert meta["reference_files"]["ke08"].startswith("f-src/mod_linfe.f90")


def _flatten(uu):
    nm, _, nl = uu.shape
    flat = np.zeros((nl, nl))
    for k in range(3):
        for l in range(nm):
            flat[k * nm + l] = uu[l, k]
    return flat


def test_quadratic_boundary_modes_equal_reference_table(orc):
    """init_displ_hexe20 (mod_write_deck.f90:118-279), parsed with Fortran's literal kinds."""
    assert np.array_equal(orc.boundary_modes20(1e-6), np.load(GOLDEN / "uu_hexe20_eps1e-6.npy"))


def test_quadratic_loadcase_matrix_against_reference_table(orc):
    """init_loadcase_el_order_quad (mod_struct_calcmat.f90:1780-2028) as written is singular;
    the oracle's matrix differs from it exactly at the table's typing defects."""
    e = 1e-6
    vv = orc.loadcase_matrix_quad(e)
    table = np.load(GOLDEN / "vv_quad_table_eps1e-6.npy")
    st = np.load(GOLDEN / "vv_quad_statements_eps1e-6.npz")
    labels, nvals, values = st["labels"], st["nvals"], st["values"]
    # (1) the statement in row 49's place is labelled 59 and a later vv(59,:) overwrites it,
    # so the table's row 49 is zero and the table is singular
    assert labels[48] == 59 and labels[58] == 59 and list(labels).count(49) == 0
    assert not table[48].any() and np.linalg.matrix_rank(table) == 59
    # (2) row 54's statement has 61 values, the surplus one a trailing zero
    assert nvals[53] == 61 and values[53, 60] == 0.0 and (nvals[np.arange(60) != 53] == 60).all()
    # (3) the intended table: row 49 from the mislabelled statement, entries written without
    # the factor e (22 of them, one in the mislabelled row; all |v| >= 0.5, where every
    # e-scaled entry is below 1e-5)
    intended = table.copy()
    intended[48] = values[48, :60]
    bare = np.abs(intended) > 1e-3
    assert bare.sum() == 22
    intended[bare] *= e
    # (4) with those repairs every entry agrees
    assert np.array_equal(intended, vv)
    # (5) and it is the flattened boundary-mode table except for the two entries the table
    # writes 0.9_rk*e where the boundary modes multiply eps by the single-precision .9
    flat = _flatten(orc.boundary_modes20(e))
    assert sorted(map(tuple, np.argwhere(flat != vv))) == [(9, 48), (58, 11)]
    assert np.abs(flat - vv).max() < 1e-7 * e
    assert abs(np.linalg.cond(vv) - 19.3518) < 1e-3


def test_quadratic_modes_reproduce_affine_fields():
    """Load cases 1-6 of the quadratic macro element are the six affine strain modes: at every
    corner and mid-edge node their value is the linear field the 8-node modes interpolate."""
    uu20 = np.load(GOLDEN / "uu_hexe20_eps1e-6.npy")
    uu8 = np.load(GOLDEN / "uu_hexe8_eps1e-6.npy")
    corners = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                        [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
    # ANSYS mid-edge nodes 9-20 (phi_NN_hexe20, mod_linfe.f90:851-866)
    mids = np.array([[0, -1, -1], [1, 0, -1], [0, 1, -1], [-1, 0, -1], [0, -1, 1], [1, 0, 1],
                     [0, 1, 1], [-1, 0, 1], [-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], float)
    pts = np.vstack([corners, mids])
    N8 = np.prod(0.5 * (1 + pts[:, None, :] * corners[None, :, :]), axis=2)   # (20 points, 8)
    for lc in range(6):
        assert np.allclose(N8 @ uu8[:, :, lc], uu20[:, :, lc], rtol=0, atol=1e-20)
