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


def _fake_results(n, seed=5):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        r = {"domain_number": 10 + i, "ne": int(rng.integers(1, 1000)), "nn": int(rng.integers(1, 1000)),
             "iters": rng.integers(1, 500, 24), "ff": rng.standard_normal((24, 24)),
             "kmacro": rng.standard_normal((24, 24)), "sym_k": rng.random(), "c": rng.standard_normal((6, 6)),
             "sym_c": rng.random(), "ee": rng.standard_normal((6, 6)), "sym_ee": rng.random(), "density": rng.random()}
        for k in ("cr1", "cr2"):
            r[k] = {"angle": rng.random(), "n": rng.standard_normal(3), "aa": rng.standard_normal((3, 3)),
                    "ee": rng.standard_normal((6, 6))}
        out.append(r)
    return out


def test_result_tree_roundtrip(dtc, tmp_path):
    """The 24-leaf result record of f-src_main/dtc.f90:738-777 written as a PureDat tree reads back
    per domain, matrices column-major (the reference's reshape order)."""
    pd = dtc.puredat
    res = _fake_results(3)
    t = pd.write_result_tree(tmp_path / "batch.head", res, start_time=1.5, duration=0.25,
                             decomposition={"x_D": np.array([20, 20, 20]), "delta": np.array([0.05, 0.05, 0.05])})
    branch = [b for b in t.root.branches if b.desc == "Averaged Material Properties"][0]
    assert [(lf.desc, lf.dat_ty, lf.dat_no) for lf in branch.leaves] == \
        [(d, ty, per * 3) for d, ty, per in pd.RESULT_LEAVES]
    # the head text re-parses to the same tree (format of the reference's writer)
    assert pd.head_text(pd.read_head(tmp_path / "batch.head")) == (tmp_path / "batch.head").read_text()
    back = pd.read_result_tree(tmp_path / "batch.head")
    for r, b in zip(res, back):
        assert b["Domain number"][0] == r["domain_number"]
        assert (b["Collected logs"] == r["iters"]).all()
        assert np.array_equal(b["Domain forces"], r["ff"].reshape(-1, order="F"))
        assert np.array_equal(b["Effective stiffness"].reshape(6, 6, order="F"), r["c"])
        assert np.array_equal(b["Final coordinate system CR_2"].reshape(3, 3, order="F"), r["cr2"]["aa"])
        assert b["Start Time"][0] == 1.5 and b["Duration"][0] == 0.25
        assert b["Effective density"][0] == r["density"]
    assert np.array_equal(t.read("x_D"), [20, 20, 20])


def test_result_leaf_names_match_shipped_results_branch(dtc):
    """Every leaf of the reference's shipped (older, 18-leaf) result branch is one of the 24
    leaves written here, with the same type and the same values per domain."""
    pd = dtc.puredat
    root = pd.read_head(GOLDEN / "puredat" / "solid_cube_Hex08.head")
    shipped = [b for b in root.branches if b.desc == "Averaged Material Properties"][0]
    ours = {d: (ty, per) for d, ty, per in pd.RESULT_LEAVES}
    for lf in shipped.leaves:
        assert lf.desc in ours, lf.desc
        assert ours[lf.desc][0] == lf.dat_ty
        assert lf.dat_no % ours[lf.desc][1] == 0


@pytest.mark.gpu
def test_result_tree_of_a_solve(dtc, tmp_path):
    syn = dtc.synth
    doms = [dtc.Domain(syn.bone_volume((10, 10, 10), b, syn.seed_for(8, 40 + i)), E=syn.E_CONST, nu=syn.NU,
                       delta=syn.DELTA, domain_number=7 + i) for i, b in enumerate((0.4, 0.55))]
    with dtc.Solver(precision="fp64", rtol=1e-8, rotation_search=True) as s:
        res = s.solve(doms)
        ms = s.stats()["ms_solve"]
    dtc.puredat.write_result_tree(tmp_path / "r.head", res, duration=ms / 1e3)
    back = dtc.puredat.read_result_tree(tmp_path / "r.head")
    for r, b in zip(res, back):
        assert b["Domain number"][0] == r["domain_number"]
        assert (b["Number of Elements"][0], b["Number of Nodes"][0]) == (r["ne"], r["nn"])
        assert np.array_equal(b["Averaged Effective stiffness"].reshape(6, 6, order="F"), r["ee"])
        assert np.array_equal(b["Optimized Effective stiffness CR_1"].reshape(6, 6, order="F"), r["cr1"]["ee"])
        assert b["Rotation Angle CR_2"][0] == r["cr2"]["angle"]
