"""PureDat trees (the reference's on-disk format, f-src/mod_puredat.f90): the head parser and
writer reproduce the reference's shipped head files byte for byte; scalar volumes written here
read back domain by domain with the reference's row positions (mod_struct_preprocess.f90:225-242)
and the reference's decomposition (synth.volume_domains)."""
import numpy as np
import pytest

from conftest import GOLDEN

HEADS = sorted((GOLDEN / "puredat").glob("*.head"))


@pytest.mark.parametrize("head", HEADS, ids=[h.name for h in HEADS])
def test_head_roundtrip_is_byte_exact(dtc, head):
    pd = dtc.puredat
    root = pd.read_head(head)
    assert pd.head_text(root) == head.read_text()


def test_shipped_scalar_volume_head(dtc):
    pd = dtc.puredat
    root = pd.read_head(GOLDEN / "puredat" / "SC00-0_tc_Dev_BinDecomp_isotropic-HEX08.head")
    assert root.streams == [0, 0, 9267, 0, 6, 12, 0]
    sd = root.leaves[0]
    assert (sd.desc, sd.dat_no, sd.dat_ty, sd.lbound, sd.ubound) == ("Scalar data", 21 ** 3, 3, 1, 9261)
    assert [lf.desc for lf in root.leaves] == ["Scalar data", "Number of voxels per direction", "Origin",
                                              "Grid spacings", "Origin shift against global coordinate system",
                                              "Field content description"]


def test_shipped_results_head(dtc):
    pd = dtc.puredat
    root = pd.read_head(GOLDEN / "puredat" / "solid_cube_Hex08.head")
    names = [b.desc for b in root.branches]
    assert names == ["Input parameters", "Global domain decomposition", "Averaged Material Properties"]
    res = root.branches[2]
    ff = [lf for lf in res.leaves if lf.desc == "Domain forces"][0]
    assert (ff.dat_no, ff.dat_ty) == (576, 5) and ff.ubound - ff.lbound + 1 == 576


@pytest.mark.parametrize("dtype", [np.int8, np.int16, np.int32])
def test_scalar_volume_domains_roundtrip(dtc, tmp_path, dtype):
    pd, syn = dtc.puredat, dtc.synth
    rng = np.random.default_rng(4)
    hi = {np.int8: 120, np.int16: 30000, np.int32: 2 ** 30}[dtype]
    vol = rng.integers(-hi, hi, size=(22, 26, 34)).astype(dtype)   # z, y, x
    t = pd.write_scalar_tree(tmp_path / "vol.head", vol, (0.05, 0.05, 0.05))
    assert t.volume_info() == ((34, 26, 22), (0.05, 0.05, 0.05))
    assert pd.head_text(pd.read_head(tmp_path / "vol.head")) == (tmp_path / "vol.head").read_text()
    got = list(pd.puredat_domains(tmp_path / "vol.head", 8))
    want = syn.volume_domains(vol, 8)
    assert len(got) == len(want) == 4 * 3 * 2
    for (d, xa, phi, delta), (d2, xa2, phi2) in zip(got, want):
        assert (d, tuple(xa)) == (d2, tuple(xa2)) and delta == (0.05, 0.05, 0.05)
        assert phi.dtype == np.dtype(dtype) and np.array_equal(phi, phi2)
    # the reference's row positions (1-based bytes) into the stream file
    raw = (tmp_path / f"vol.int{np.dtype(dtype).itemsize}.st").read_bytes()
    lb = t.find("Scalar data").lbound
    vd = (34, 26, 22)
    d, xa, phi, _ = got[13]
    m = np.dtype(dtype).itemsize
    for z in range(xa[2], xa[2] + 8):
        for y in range(xa[1], xa[1] + 8):
            pos_f = (vd[0] * vd[1] * (z - 1) + vd[0] * (y - 1) + (xa[0] - 1) + lb - 1) * m + 1
            row = np.frombuffer(raw[pos_f - 1: pos_f - 1 + 8 * m], dtype=dtype)
            assert np.array_equal(row, phi[z - xa[2], y - xa[1]])


def test_domain_outside_volume_rejected(dtc, tmp_path):
    pd = dtc.puredat
    t = pd.write_scalar_tree(tmp_path / "v.head", np.zeros((10, 10, 10), np.int16), (0.1, 0.1, 0.1))
    with pytest.raises(ValueError):
        t.read_domain((5, 1, 1), (8, 8, 8))
