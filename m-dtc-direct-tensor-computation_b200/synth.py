"""Seeded synthetic trabecular-bone volumes (no CT data travels with this project).

Recipe: white noise N(0,1) -> Gaussian filter (sigma = 2 voxels, reflect) -> threshold at
the (1 - BV/TV) quantile -> keep the largest 6-connected bone component -> bone gray values
uniform in [20000, 30000], marrow 0 (int16; the reference reads TYPE_RAW ik2 signed).
Per-voxel modulus E = 5000 + 1.5 (g - 20000) MPa, i.e. [5000, 20000].
"""
import numpy as np
from scipy import ndimage

DELTA = 0.05          # mm voxel edge
NU = 0.3
LLIMIT = 1            # BINARIZE_LO
RVE_STRAIN = 1e-6
E_CONST = 5600.0      # YOUNG_MODULUS of the reference's own test metas


def seed_for(config, index):
    return 1_000_003 * config + index


def bone_volume(shape, bvtv, seed, sigma=2.0):
    """int16 gray volume indexed [z, y, x] (x fastest)."""
    rng = np.random.default_rng(seed)
    field = ndimage.gaussian_filter(rng.standard_normal(shape), sigma=sigma, mode="reflect")
    thr = np.quantile(field, 1.0 - bvtv)
    bone = field > thr
    lab, n = ndimage.label(bone)
    if n > 1:
        sizes = np.bincount(lab.ravel())
        sizes[0] = 0
        bone = lab == np.argmax(sizes)
    gray = np.zeros(shape, np.int16)
    gray[bone] = rng.integers(20000, 30001, size=int(bone.sum())).astype(np.int16)
    return gray


def modulus_of_gray(gray):
    """Per-voxel Young's modulus (float32 MPa) from gray values; 0 for marrow."""
    g = gray.astype(np.float64)
    return np.where(g > 0, 5000.0 + 1.5 * (g - 20000.0), 0.0).astype(np.float32)


def volume_domains(gray, L):
    """Domain decomposition of a volume with the reference's 1-voxel frame
    (mod_decomp.f90:298-301, mod_struct_preprocess.f90:85-98): nn_D = (vdim - 2) / L
    domains per axis, domain (i,j,k) covers voxels xa_n = L*(i,j,k) + 2 .. + L - 1
    (1-based), numbered d = i + j*nn_D1 + k*nn_D1*nn_D2."""
    vz, vy, vx = gray.shape
    nd = [(vx - 2) // L, (vy - 2) // L, (vz - 2) // L]
    out = []
    for k in range(nd[2]):
        for j in range(nd[1]):
            for i in range(nd[0]):
                xa = (L * i + 2, L * j + 2, L * k + 2)
                sub = gray[xa[2] - 1: xa[2] - 1 + L, xa[1] - 1: xa[1] - 1 + L, xa[0] - 1: xa[0] - 1 + L]
                out.append((i + j * nd[0] + k * nd[0] * nd[1], xa, np.ascontiguousarray(sub)))
    return out
