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
