"""ctypes binding of the FP64 CPU oracle (oracle/liborc_dtc.so) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs use this
module, and only as the checker.  The product library never imports it.
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liborc_dtc.so"

ORC_OK, ORC_EMPTY, ORC_NO_STRUCTURE, ORC_FEW_NODES, ORC_MAX_IT, ORC_BREAKDOWN, ORC_NONFINITE = range(7)


class OrcIn(C.Structure):
    _fields_ = [
        ("L", C.c_int64 * 3), ("xa_n", C.c_int64 * 3), ("llimit", C.c_int64),
        ("nen", C.c_int32), ("rotation", C.c_int32),
        ("delta", C.c_double * 3), ("phdsize", C.c_double * 3),
        ("E", C.c_double), ("nu", C.c_double), ("rve_strain", C.c_double),
        ("rtol", C.c_double), ("max_it", C.c_int64),
        ("phi", C.POINTER(C.c_int32)), ("E_voxel", C.POINTER(C.c_float)),
        ("macro_order", C.c_int32), ("pad_", C.c_int32),
    ]


class OrcOut(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("ne", C.c_int64), ("nn", C.c_int64), ("nb", C.c_int64),
        ("iters", C.c_int64 * 60),
        ("ff", C.c_double * 3600), ("kmacro", C.c_double * 3600), ("sym_k", C.c_double),
        ("c", C.c_double * 36), ("sym_c", C.c_double),
        ("ee", C.c_double * 36), ("sym_ee", C.c_double),
        ("cr1_angle", C.c_double), ("cr1_n", C.c_double * 3), ("cr1_aa", C.c_double * 9),
        ("cr1_ee", C.c_double * 36), ("cr1_crit", C.c_double),
        ("cr2_angle", C.c_double), ("cr2_n", C.c_double * 3), ("cr2_aa", C.c_double * 9),
        ("cr2_ee", C.c_double * 36), ("cr2_crit", C.c_double),
        ("cr1_iters", C.c_int32), ("cr2_iters", C.c_int32),
        ("density", C.c_double),
        ("cap_elems", C.c_int64), ("cap_nodes", C.c_int64),
        ("elems", C.POINTER(C.c_int64)), ("elem_voxel", C.POINTER(C.c_int64)),
        ("nodes", C.POINTER(C.c_double)),
        ("bnode_ids", C.POINTER(C.c_int64)), ("bnode_vals", C.POINTER(C.c_double)),
        ("displ", C.POINTER(C.c_double)), ("force", C.POINTER(C.c_double)),
        ("cr1_ang", C.c_int64 * 3), ("cr2_ang", C.c_int64 * 3),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        _lib.orc_solve_domain.argtypes = [C.POINTER(OrcIn), C.POINTER(OrcOut)]
        _lib.orc_mesh_domain.argtypes = [C.POINTER(OrcIn), C.POINTER(OrcOut)]
        _lib.orc_solve_batch.argtypes = [C.POINTER(OrcIn), C.POINTER(OrcOut), C.c_int64, C.c_int32]
        _lib.orc_element_stiffness.argtypes = [C.c_int32, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double)]
        _lib.orc_boundary_modes.argtypes = [C.c_double, C.POINTER(C.c_double)]
        _lib.orc_loadcase_matrix.argtypes = [C.c_double, C.POINTER(C.c_double)]
        _lib.orc_boundary_modes20.argtypes = [C.c_double, C.POINTER(C.c_double)]
        _lib.orc_loadcase_matrix_quad.argtypes = [C.c_double, C.POINTER(C.c_double)]
        _lib.orc_rotation_search.argtypes = [C.POINTER(C.c_double), C.POINTER(OrcOut)]
    return _lib


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int64))


def element_stiffness(nen, E, a, nu):
    nd = 3 * nen
    ke = np.zeros((nd, nd), order="F")
    lib().orc_element_stiffness(nen, E, a, nu, _dptr(ke))
    return ke


def boundary_modes(eps=1e-6):
    uu = np.zeros((8, 3, 24), order="F")
    lib().orc_boundary_modes(eps, _dptr(uu))
    return uu


def loadcase_matrix(eps=1e-6):
    vv = np.zeros((24, 24), order="F")
    lib().orc_loadcase_matrix(eps, _dptr(vv))
    return vv


def boundary_modes20(eps=1e-6):
    uu = np.zeros((20, 3, 60), order="F")
    lib().orc_boundary_modes20(eps, _dptr(uu))
    return uu


def loadcase_matrix_quad(eps=1e-6):
    vv = np.zeros((60, 60), order="F")
    lib().orc_loadcase_matrix_quad(eps, _dptr(vv))
    return vv


class Domain:
    """One domain's input, held with its backing numpy arrays alive."""

    def __init__(self, phi, *, llimit=1, nen=8, delta=0.05, phdsize=None, E=5600.0, nu=0.3,
                 rve_strain=1e-6, rtol=1e-10, max_it=500000, xa_n=(2, 2, 2), rotation=False,
                 E_voxel=None, macro_order=1):
        phi = np.asarray(phi)
        assert phi.ndim == 3, "phi is indexed [z, y, x] (x fastest in memory)"
        self.phi = np.ascontiguousarray(phi, dtype=np.int32)
        L = (phi.shape[2], phi.shape[1], phi.shape[0])
        self.E_voxel = None if E_voxel is None else np.ascontiguousarray(E_voxel, dtype=np.float32)
        d = (delta,) * 3 if np.isscalar(delta) else tuple(delta)
        ph = tuple(L[i] * d[i] for i in range(3)) if phdsize is None else (
            (phdsize,) * 3 if np.isscalar(phdsize) else tuple(phdsize))
        self.s = OrcIn()
        self.s.L[:] = L
        self.s.xa_n[:] = xa_n
        self.s.llimit = llimit
        self.s.nen = nen
        self.s.rotation = int(rotation)
        self.s.delta[:] = d
        self.s.phdsize[:] = ph
        self.s.E, self.s.nu, self.s.rve_strain = E, nu, rve_strain
        self.s.rtol, self.s.max_it = rtol, max_it
        self.s.phi = self.phi.ctypes.data_as(C.POINTER(C.c_int32))
        self.s.E_voxel = (self.E_voxel.ctypes.data_as(C.POINTER(C.c_float))
                          if self.E_voxel is not None else C.POINTER(C.c_float)())
        self.s.macro_order = int(macro_order)
        self.L = L
        self.nen = nen
        self.nl = 60 if macro_order == 2 else 24


def _out_struct(dom, with_arrays):
    o = OrcOut()
    keep = {}
    if with_arrays:
        L = dom.L
        me = L[0] * L[1] * L[2]
        if dom.nen == 8:
            mn = (L[0] + 1) * (L[1] + 1) * (L[2] + 1)
        else:
            mn = (2 * L[0] + 1) * (2 * L[1] + 1) * (2 * L[2] + 1)
        keep["elems"] = np.zeros(dom.nen * me, np.int64)
        keep["elem_voxel"] = np.zeros(me, np.int64)
        keep["nodes"] = np.zeros(3 * mn)
        keep["bnode_ids"] = np.zeros(mn, np.int64)
        keep["bnode_vals"] = np.zeros(dom.nl * 3 * mn)
        keep["displ"] = np.zeros(dom.nl * 3 * mn)
        keep["force"] = np.zeros(dom.nl * 3 * mn)
        o.cap_elems, o.cap_nodes = me, mn
        o.elems, o.elem_voxel = _iptr(keep["elems"]), _iptr(keep["elem_voxel"])
        o.nodes = _dptr(keep["nodes"])
        o.bnode_ids, o.bnode_vals = _iptr(keep["bnode_ids"]), _dptr(keep["bnode_vals"])
        o.displ, o.force = _dptr(keep["displ"]), _dptr(keep["force"])
    return o, keep


def _result(dom, o, keep):
    nl = dom.nl if dom is not None else 24
    r = {
        "status": o.status, "ne": o.ne, "nn": o.nn, "nb": o.nb,
        "iters": np.array(o.iters[:nl]),
        "ff": np.array(o.ff[: nl * nl]).reshape(nl, nl, order="F"),
        "kmacro": np.array(o.kmacro[: nl * nl]).reshape(nl, nl, order="F"),
        "sym_k": o.sym_k, "c": np.array(o.c[:]).reshape(6, 6, order="F"), "sym_c": o.sym_c,
        "ee": np.array(o.ee[:]).reshape(6, 6, order="F"), "sym_ee": o.sym_ee,
        "density": o.density,
    }
    for k in ("cr1", "cr2"):
        r[k] = {
            "angle": getattr(o, k + "_angle"), "n": np.array(getattr(o, k + "_n")[:]),
            "aa": np.array(getattr(o, k + "_aa")[:]).reshape(3, 3, order="F"),
            "ee": np.array(getattr(o, k + "_ee")[:]).reshape(6, 6, order="F"),
            "crit": getattr(o, k + "_crit"), "iters": getattr(o, k + "_iters"),
            "ang": np.array(getattr(o, k + "_ang")[:], dtype=np.int64),
        }
    if keep:
        ne, nn, nb = o.ne, o.nn, o.nb
        r["elems"] = keep["elems"][: dom.nen * ne].reshape(ne, dom.nen)
        r["elem_voxel"] = keep["elem_voxel"][:ne]
        r["nodes"] = keep["nodes"][: 3 * nn].reshape(nn, 3)
        r["bnode_ids"] = keep["bnode_ids"][:nb]
        r["bnode_vals"] = keep["bnode_vals"][: nl * 3 * nb].reshape(nl, 3 * nb, order="F")
        r["displ"] = keep["displ"][: nl * 3 * nn].reshape(nl, 3 * nn)
        r["force"] = keep["force"][: nl * 3 * nn].reshape(nl, 3 * nn)
    return r


def solve_domain(dom, with_arrays=False):
    o, keep = _out_struct(dom, with_arrays)
    lib().orc_solve_domain(C.byref(dom.s), C.byref(o))
    return _result(dom, o, keep)


def mesh_domain(dom):
    o, keep = _out_struct(dom, True)
    lib().orc_mesh_domain(C.byref(dom.s), C.byref(o))
    return _result(dom, o, keep)


def solve_batch(doms, nthreads=0):
    n = len(doms)
    ins = (OrcIn * n)(*[d.s for d in doms])
    outs = (OrcOut * n)()
    lib().orc_solve_batch(ins, outs, n, nthreads or (os.cpu_count() or 1))
    return [_result(d, outs[i], {}) for i, d in enumerate(doms)]


def rotation_search(ee):
    ee = np.asfortranarray(np.asarray(ee, dtype=np.float64))
    o = OrcOut()
    lib().orc_rotation_search(_dptr(ee), C.byref(o))
    return _result(None, o, {})
