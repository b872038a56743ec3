"""ctypes declarations of include/dtc.h and loading of the in-tree libdtc.so.

The library is the product: if libdtc.so is missing or cannot be loaded this module
raises, it never falls back to a CPU implementation.
"""
import ctypes as C

import numpy as np
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libdtc.so"
ABI_VERSION = 2

DTC_OK, DTC_ERR_INVALID_ARGUMENT, DTC_ERR_CUDA, DTC_ERR_OUT_OF_MEMORY, DTC_ERR_NO_DEVICE, \
    DTC_ERR_ABI_MISMATCH, DTC_ERR_INTERNAL = range(7)
STATUS_NAMES = {0: "OK", 1: "INVALID_ARGUMENT", 2: "CUDA", 3: "OUT_OF_MEMORY", 4: "NO_DEVICE",
                5: "ABI_MISMATCH", 6: "INTERNAL"}
DOMAIN_OK, DOMAIN_EMPTY, DOMAIN_NO_STRUCTURE, DOMAIN_FEW_NODES, DOMAIN_MAX_IT, DOMAIN_BREAKDOWN, \
    DOMAIN_NONFINITE = range(7)
HEX08, HEX20 = 8, 20
PREC_FP64, PREC_MIXED = 0, 1


class Options(C.Structure):
    _fields_ = [
        ("abi_version", C.c_int32), ("precision", C.c_int32), ("rtol", C.c_double),
        ("max_it", C.c_int64), ("inner_rtol", C.c_double), ("max_refine", C.c_int32),
        ("rotation_search", C.c_int32), ("device", C.c_int32), ("host_threads", C.c_int32),
        ("keep_displacements", C.c_int32), ("profile_kernels", C.c_int32),
        ("mixed_matvec", C.c_int32), ("inner_precond", C.c_int32),
        ("tensor_estimator", C.c_int32), ("chunk_domains", C.c_int32), ("graph_chunks", C.c_int32),
        ("tc_wait_spins", C.c_int32), ("device_mesher", C.c_int32), ("macro_order", C.c_int32),
    ]


class DomainIn(C.Structure):
    _fields_ = [
        ("L", C.c_int64 * 3), ("xa_n", C.c_int64 * 3), ("domain_number", C.c_int64),
        ("elem_type", C.c_int32), ("phi_type", C.c_int32), ("phi", C.c_void_p),
        ("llimit", C.c_int64), ("E_voxel", C.POINTER(C.c_float)),
        ("delta", C.c_double * 3), ("phdsize", C.c_double * 3),
        ("E", C.c_double), ("nu", C.c_double), ("rve_strain", C.c_double),
    ]


class Macro2Out(C.Structure):
    _fields_ = [("iters", C.c_int64 * 60), ("relres", C.c_double * 60), ("ff", C.c_double * 3600),
                ("kmacro", C.c_double * 3600)]


class DomainOut(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("refine_steps", C.c_int32), ("domain_number", C.c_int64),
        ("ne", C.c_int64), ("nn", C.c_int64), ("nb", C.c_int64), ("n_free_dof", C.c_int64),
        ("iters", C.c_int64 * 24), ("relres", C.c_double * 24),
        ("ff", C.c_double * 576), ("kmacro", C.c_double * 576), ("sym_k", C.c_double),
        ("c", C.c_double * 36), ("sym_c", C.c_double), ("ee", C.c_double * 36), ("sym_ee", C.c_double),
        ("cr1_angle", C.c_double), ("cr1_n", C.c_double * 3), ("cr1_aa", C.c_double * 9),
        ("cr1_ee", C.c_double * 36), ("cr1_crit", C.c_double),
        ("cr2_angle", C.c_double), ("cr2_n", C.c_double * 3), ("cr2_aa", C.c_double * 9),
        ("cr2_ee", C.c_double * 36), ("cr2_crit", C.c_double),
        ("cr1_iters", C.c_int32), ("cr2_iters", C.c_int32), ("density", C.c_double),
        ("displ", C.POINTER(C.c_double)), ("force", C.POINTER(C.c_double)),
        ("macro2", C.POINTER(Macro2Out)),
    ]


def numpy_dtype(struct):
    """numpy structured dtype with the field offsets of a ctypes Structure (pointers as uintp)."""
    names, formats, offsets = [], [], []
    scalar = {C.c_int32: "<i4", C.c_int64: "<i8", C.c_double: "<f8", C.c_float: "<f4", C.c_char: "S1"}
    for name, ct in struct._fields_:
        names.append(name)
        offsets.append(getattr(struct, name).offset)
        if hasattr(ct, "_length_") and hasattr(ct, "_type_") and ct._type_ in scalar:
            formats.append((scalar[ct._type_], (ct._length_,)))
        elif ct in scalar:
            formats.append(scalar[ct])
        else:   # pointer
            formats.append("<u8")
    return np.dtype({"names": names, "formats": formats, "offsets": offsets, "itemsize": C.sizeof(struct)})


class KernelStats(C.Structure):
    _fields_ = [("name", C.c_char * 32), ("launches", C.c_int64), ("ms_total", C.c_double),
                ("bytes_per_launch", C.c_double), ("flops_per_launch", C.c_double)]


class MeshOut(C.Structure):
    _fields_ = [
        ("ne", C.c_int64), ("nn", C.c_int64), ("nb", C.c_int64),
        ("status", C.c_int32), ("last_elem_partial", C.c_int32),
        ("cap_elems", C.c_int64), ("cap_nodes", C.c_int64),
        ("elems", C.POINTER(C.c_int64)), ("nodes", C.POINTER(C.c_double)),
        ("bnode_ids", C.POINTER(C.c_int64)), ("bnode_vals", C.POINTER(C.c_double)),
        ("macro_order", C.c_int32), ("pad_", C.c_int32),
    ]


# every symbol include/dtc.h declares, with its signature
SIGNATURES = {
    "dtc_abi_version": (C.c_int32, []),
    "dtc_default_options": (None, [C.POINTER(Options)]),
    "dtc_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(Options)]),
    "dtc_destroy": (C.c_int, [C.c_void_p]),
    "dtc_solve_batch": (C.c_int, [C.c_void_p, C.POINTER(DomainIn), C.c_int64, C.POINTER(DomainOut)]),
    "dtc_mesh_domain": (C.c_int, [C.POINTER(DomainIn), C.POINTER(MeshOut)]),
    "dtc_mesh_batch": (C.c_int, [C.c_void_p, C.POINTER(DomainIn), C.c_int64, C.POINTER(MeshOut)]),
    "dtc_energy_grad": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.POINTER(C.c_float)), C.c_int64]),
    "dtc_get_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_double)]),
    "dtc_element_stiffness": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "dtc_get_kernel_stats": (C.c_int, [C.c_void_p, C.POINTER(KernelStats), C.c_int32, C.POINTER(C.c_int32)]),
    "dtc_solve_batch_device_moduli": (C.c_int, [C.c_void_p, C.POINTER(DomainIn), C.c_int64, C.POINTER(DomainOut),
                                                C.POINTER(C.c_void_p)]),
    "dtc_energy_grad_device": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_void_p), C.c_int64]),
    "dtc_rotation_search": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_int64, C.POINTER(DomainOut)]),
    "dtc_rotation_search_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.c_void_p]),
    "dtc_last_error": (C.c_char_p, [C.c_void_p]),
}

_lib = None


def load():
    """Load libdtc.so (built in-tree by __graft_entry__.build() / make)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` "
                           "(or __graft_entry__.build()); there is no fallback implementation")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.dtc_abi_version() != ABI_VERSION:
        raise RuntimeError("libdtc.so ABI version mismatch")
    _lib = lib
    return lib


class DTCError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dtc error {STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code
