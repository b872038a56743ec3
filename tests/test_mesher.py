"""Bit-exact element order, node numbering and constrained-node lists of the library's host
mesher (dtc_mesh_domain) against the oracle's literal restatement of gen_quadmesh_from_phi
and generate_boundaries."""
import numpy as np
import pytest


def compare(dtc, orc, phi, nen=8, macro_order=1, **kw):
    d = dtc.Domain(phi, elem_type=nen, **kw)
    od = orc.Domain(phi, nen=nen, macro_order=macro_order, **kw)
    m = dtc.mesh_domain(d, macro_order=macro_order)
    r = orc.mesh_domain(od)
    assert m["status"] == r["status"]
    if r["status"] == 0:
        assert (m["ne"], m["nn"], m["nb"]) == (r["ne"], r["nn"], r["nb"])
        assert np.array_equal(m["elems"], r["elems"])
        assert np.array_equal(m["nodes"], r["nodes"])
        assert np.array_equal(m["bnode_ids"], r["bnode_ids"])
        assert np.array_equal(m["bnode_vals"], r["bnode_vals"])
    return m, r


@pytest.mark.parametrize("nen", [8, 20])
def test_random_volumes(dtc, orc, nen):
    rng = np.random.default_rng(11 + nen)
    for _ in range(120 if nen == 8 else 40):
        L = rng.integers(1, 9, size=3)
        p = rng.random() * 0.7
        phi = (rng.random((L[2], L[1], L[0])) < p).astype(np.int16) * int(rng.integers(1, 30000))
        compare(dtc, orc, phi, nen=nen, delta=0.05, xa_n=tuple(int(v) for v in rng.integers(1, 40, 3)))


@pytest.mark.parametrize("nen", [8, 20])
def test_quadratic_macro_boundary_values(dtc, orc, nen):
    """Macro order 2: the 60 prescribed values of every constrained node (determine_prescribed_displ
    with init_displ_hexe20 and phi_NN_hexe20, mod_write_deck.f90:22-51,118-279) bit for bit."""
    rng = np.random.default_rng(5 + nen)
    for _ in range(12):
        L = rng.integers(2, 8, size=3)
        phi = (rng.random((L[2], L[1], L[0])) < 0.6).astype(np.int16) * 1000
        m, r = compare(dtc, orc, phi, nen=nen, macro_order=2, delta=0.05,
                       xa_n=tuple(int(v) for v in rng.integers(1, 40, 3)))
        if r["status"] == 0:
            assert m["bnode_vals"].shape == (60, 3 * m["nb"])


@pytest.mark.parametrize("dtype", [np.int8, np.int16, np.int32])
def test_gray_types_and_threshold(dtc, orc, dtype):
    rng = np.random.default_rng(3)
    phi = rng.integers(-100, 100, size=(6, 7, 5)).astype(dtype)
    compare(dtc, orc, phi, llimit=20)


def test_floating_island_is_dropped(dtc, orc):
    phi = np.zeros((9, 9, 9), np.int16)
    phi[0, :, :] = 100          # slab on the bottom face: touches the bounding box
    phi[8, :, :] = 100          # top slab
    phi[:, 0, 0] = 100          # pillar joining them
    phi[4, 4, 4] = 100          # isolated voxel inside: dropped
    m, r = compare(dtc, orc, phi)
    assert m["ne"] == int((phi > 0).sum()) - 1


def test_region_touching_only_mesh_bbox_is_kept(dtc, orc):
    phi = np.zeros((8, 8, 8), np.int16)
    phi[2:6, 2:6, 2] = 100      # bone bounding box z = 2..5 (inside the domain box)
    phi[2:6, 3, 4] = 100        # a second region touching the bone bbox faces
    m, r = compare(dtc, orc, phi)
    assert m["ne"] == int((phi > 0).sum())
    assert m["nb"] == 0         # nothing on the domain box: no constrained node


def test_empty_domain(dtc, orc):
    phi = np.zeros((5, 5, 5), np.int16)
    m, r = compare(dtc, orc, phi)
    assert m["status"] == dtc.DOMAIN_EMPTY


def test_tc01_orthotropic_domain0_is_empty(dtc, orc):
    """TC01 orthotropic (regression/f-src/create_testcase.f90:101-103): two orthogonal bars at
    voxels 56-65 of a 100^3 volume; domain 0 (50^3 from voxel 2) contains no bone."""
    vol = np.zeros((100, 100, 100), np.int16)
    vol[:, 55:65, 55:65] = 14250
    vol[55:65, 55:65, :] = 14250
    dom = vol[1:51, 1:51, 1:51]
    m, r = compare(dtc, orc, dom, xa_n=(2, 2, 2), delta=0.01)
    assert m["status"] == dtc.DOMAIN_EMPTY


def test_numbering_first_appearance(dtc):
    phi = np.ones((1, 1, 2), np.int16)    # two voxels along x
    m = dtc.mesh_domain(dtc.Domain(phi, delta=1.0, xa_n=(1, 1, 1)))
    assert m["elems"].tolist() == [[1, 2, 3, 4, 5, 6, 7, 8], [2, 9, 10, 3, 6, 11, 12, 7]]
    assert m["nodes"][8].tolist() == [2.0, 0.0, 0.0]
