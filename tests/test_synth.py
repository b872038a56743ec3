"""Synthetic inputs and the reference's domain decomposition."""
import numpy as np
from scipy import ndimage


def test_bone_volume_recipe(dtc):
    syn = dtc.synth
    g = syn.bone_volume((40, 40, 40), 0.25, syn.seed_for(0, 0))
    bone = g > 0
    assert 0.15 < bone.mean() <= 0.25 + 1e-9
    lab, n = ndimage.label(bone)
    assert n == 1                                     # largest 6-connected component only
    assert g[bone].min() >= 20000 and g[bone].max() <= 30000
    assert np.array_equal(g, syn.bone_volume((40, 40, 40), 0.25, syn.seed_for(0, 0)))   # seeded
    E = syn.modulus_of_gray(g)
    assert E[bone].min() >= 5000 and E[bone].max() <= 20000 and (E[~bone] == 0).all()


def test_volume_decomposition_matches_reference_formulas(dtc):
    """62^3 volume, 20^3 domains: nn_D = (62 - 2)/20 = 3 per axis (mod_decomp.f90:301), 27
    domains; domain d = i + 3j + 9k covers voxels 20*(i,j,k) + 2 .. + 21
    (mod_struct_preprocess.f90:85-98)."""
    vol = np.arange(62 ** 3, dtype=np.int32).reshape(62, 62, 62)
    doms = dtc.synth.volume_domains(vol, 20)
    assert len(doms) == 27
    for d, xa, sub in doms:
        i, j, k = d % 3, (d // 3) % 3, d // 9
        assert xa == (20 * i + 2, 20 * j + 2, 20 * k + 2)
        assert sub.shape == (20, 20, 20)
        assert sub[0, 0, 0] == vol[xa[2] - 1, xa[1] - 1, xa[0] - 1]
    assert len(dtc.synth.volume_domains(np.zeros((60, 60, 60)), 20)) == 8   # 60^3 -> 2 per axis
