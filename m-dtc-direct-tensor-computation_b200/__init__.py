"""B200-native direct tensor computation: per-domain homogenisation of voxel bone domains.

Python mirror of the C ABI in include/dtc.h.  One call meshes, solves the 24 macro load
cases and homogenises many domains at once on one GPU, the way the reference's MPI driver
calls exec_single_domain per domain (f-src_main/struct_process.f90:1293).

    import dtc_b200 as dtc
    solver = dtc.Solver(precision="mixed", rtol=1e-8)
    results = solver.solve([dtc.Domain(phi) for phi in volumes])
    results[0]["c"]          # 6x6 effective stiffness (MPa)
"""
import ctypes as C

import numpy as np

from . import capi, puredat, synth
from .capi import (DOMAIN_BREAKDOWN, DOMAIN_EMPTY, DOMAIN_FEW_NODES, DOMAIN_MAX_IT, DOMAIN_NO_STRUCTURE,
                   DOMAIN_NONFINITE, DOMAIN_OK, HEX08, HEX20, PREC_FP64, PREC_MIXED, DTCError)

__all__ = ["Domain", "Solver", "mesh_domain", "element_stiffness", "solve_batch", "DTCError", "HEX08", "HEX20",
           "DOMAIN_OK", "DOMAIN_EMPTY", "DOMAIN_NO_STRUCTURE", "DOMAIN_FEW_NODES", "DOMAIN_MAX_IT",
           "DOMAIN_BREAKDOWN", "DOMAIN_NONFINITE"]


class Domain:
    """One control volume: gray values phi[z, y, x] plus the meta parameters the reference
    reads for it (BINARIZE_LO, SPACING, SIZE_DOMAIN, YOUNG_MODULUS, POISSON_RATIO, RVE_STRAIN,
    MICRO_ELMNT_TYPE) and its position xa_n in the volume."""

    def __init__(self, phi, *, llimit=1, elem_type=HEX08, delta=0.05, phdsize=None, E=5600.0, nu=0.3,
                 rve_strain=1e-6, xa_n=(2, 2, 2), E_voxel=None, domain_number=0):
        phi = np.asarray(phi)
        if phi.ndim != 3:
            raise ValueError("phi must be a 3-D array indexed [z, y, x]")
        if phi.dtype == np.uint16:
            if phi.size and phi.max() > 32767:
                raise ValueError("uint16 gray values above 32767 do not fit the reference's signed ik2")
            phi = phi.astype(np.int16)
        if phi.dtype not in (np.int8, np.int16, np.int32):
            phi = phi.astype(np.int32)
        self.phi = np.ascontiguousarray(phi)
        self.L = (phi.shape[2], phi.shape[1], phi.shape[0])
        self.E_voxel = None if E_voxel is None else np.ascontiguousarray(E_voxel, dtype=np.float32)
        if self.E_voxel is not None and self.E_voxel.shape != phi.shape:
            raise ValueError("E_voxel must have the shape of phi")
        d = (float(delta),) * 3 if np.isscalar(delta) else tuple(map(float, delta))
        if phdsize is None:
            ph = tuple(self.L[i] * d[i] for i in range(3))
        else:
            ph = (float(phdsize),) * 3 if np.isscalar(phdsize) else tuple(map(float, phdsize))
        self.struct = capi.DomainIn()
        s = self.struct
        s.L[:] = self.L
        s.xa_n[:] = xa_n
        s.domain_number = domain_number
        s.elem_type = elem_type
        s.phi_type = self.phi.dtype.itemsize
        s.phi = self.phi.ctypes.data
        s.llimit = llimit
        s.E_voxel = (self.E_voxel.ctypes.data_as(C.POINTER(C.c_float)) if self.E_voxel is not None
                     else C.POINTER(C.c_float)())
        s.delta[:] = d
        s.phdsize[:] = ph
        s.E, s.nu, s.rve_strain = float(E), float(nu), float(rve_strain)
        self.elem_type = elem_type


_OUT_DTYPE = capi.numpy_dtype(capi.DomainOut)


_M2_DTYPE = capi.numpy_dtype(capi.Macro2Out)


def _results(outs, keep, macro2=None):
    """Result dicts of a dtc_domain_out array: each field copied once for the whole batch, then
    per-domain rows (the 24 x 24 / 6 x 6 / 3 x 3 leaves are column-major, as in the record).
    macro2: the dtc_macro2_out array of a macro order 2 solve, whose 60-load-case leaves replace
    iters, relres, ff and kmacro."""
    raw = (C.c_char * C.sizeof(outs)).from_buffer(outs)
    a = np.frombuffer(raw, dtype=_OUT_DTYPE)
    n = len(a)
    sc = {k: a[k].tolist() for k in ("status", "refine_steps", "domain_number", "ne", "nn", "nb", "n_free_dof",
                                      "sym_k", "sym_c", "sym_ee", "density", "cr1_angle", "cr1_crit", "cr1_iters",
                                      "cr2_angle", "cr2_crit", "cr2_iters")}
    ar = {k: np.array(a[k]) for k in ("iters", "relres", "cr1_n", "cr2_n")}
    mat = {k: np.array(a[k]).reshape((n,) + shape[::-1]).transpose(0, 2, 1)
           for k, shape in (("ff", (24, 24)), ("kmacro", (24, 24)), ("c", (6, 6)), ("ee", (6, 6)),
                            ("cr1_aa", (3, 3)), ("cr1_ee", (6, 6)), ("cr2_aa", (3, 3)), ("cr2_ee", (6, 6)))}
    nl = 24
    if macro2 is not None:
        nl = 60
        m2 = np.frombuffer((C.c_char * C.sizeof(macro2)).from_buffer(macro2), dtype=_M2_DTYPE)
        ar["iters"], ar["relres"] = np.array(m2["iters"]), np.array(m2["relres"])
        for k in ("ff", "kmacro"):
            mat[k] = np.array(m2[k]).reshape(n, 60, 60).transpose(0, 2, 1)
    res = []
    for i in range(n):
        r = {k: sc[k][i] for k in ("status", "refine_steps", "domain_number", "ne", "nn", "nb", "n_free_dof",
                                    "sym_k", "sym_c", "sym_ee", "density")}
        r.update(iters=ar["iters"][i], relres=ar["relres"][i], ff=mat["ff"][i], kmacro=mat["kmacro"][i],
                 c=mat["c"][i], ee=mat["ee"][i])
        for k in ("cr1", "cr2"):
            r[k] = {"angle": sc[k + "_angle"][i], "n": ar[k + "_n"][i], "aa": mat[k + "_aa"][i],
                    "ee": mat[k + "_ee"][i], "crit": sc[k + "_crit"][i], "iters": sc[k + "_iters"][i]}
        if keep:
            nn = r["nn"]
            r["displ"] = keep[i][0][: nl * 3 * nn].reshape(nl, 3 * nn)
            r["force"] = keep[i][1][: nl * 3 * nn].reshape(nl, 3 * nn)
        res.append(r)
    return res


class Solver:
    """A handle on one GPU (dtc_create / dtc_destroy)."""

    def __init__(self, precision="fp64", rtol=1e-3, max_it=500000, inner_rtol=0.0, max_refine=12,
                 rotation_search=True, device=0, host_threads=0, keep_displacements=False,
                 profile_kernels=False, mixed_matvec="simt", inner_precond="block", estimator="reaction",
                 chunk_domains=0, graphs=True, tc_wait_spins=0, device_mesher=False, macro_order=1):
        self.lib = capi.load()
        o = capi.Options()
        self.lib.dtc_default_options(C.byref(o))
        o.precision = {"fp64": PREC_FP64, "mixed": PREC_MIXED}[precision]
        o.rtol, o.max_it, o.inner_rtol, o.max_refine = float(rtol), int(max_it), float(inner_rtol), int(max_refine)
        o.rotation_search, o.device, o.host_threads = int(bool(rotation_search)), int(device), int(host_threads)
        o.keep_displacements = int(bool(keep_displacements))
        o.profile_kernels = int(bool(profile_kernels))
        o.mixed_matvec = {"simt": 0, "tensor": 1, "auto": 2}[mixed_matvec]
        o.inner_precond = {"jacobi": 0, "block": 1, "mg": 2}[inner_precond]
        o.tensor_estimator = {"reaction": 0, "energy": 1}[estimator]
        o.chunk_domains = int(chunk_domains)
        o.graph_chunks = 0 if graphs else 1
        o.tc_wait_spins = int(tc_wait_spins)
        o.device_mesher = int(bool(device_mesher))
        o.macro_order = int(macro_order)
        self.macro_order = int(macro_order)
        self.options = o
        h = C.c_void_p()
        rc = self.lib.dtc_create(C.byref(h), C.byref(o))
        if rc != capi.DTC_OK:
            raise DTCError(rc, "dtc_create failed")
        self.handle = h

    def close(self):
        if getattr(self, "handle", None):
            self.lib.dtc_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != capi.DTC_OK:
            raise DTCError(rc, (self.lib.dtc_last_error(self.handle) or b"").decode())

    def solve(self, domains, want_fields=False):
        n = len(domains)
        ins = (capi.DomainIn * n)(*[d.struct for d in domains])
        outs = (capi.DomainOut * n)()
        m2 = self._macro2(outs)
        nl = 60 if m2 is not None else 24
        keep = []
        if want_fields:
            for i, d in enumerate(domains):
                m = 1 if d.elem_type == HEX08 else 2   # HEX20 nodes live on the doubled grid
                cap = nl * 3 * (m * d.L[0] + 1) * (m * d.L[1] + 1) * (m * d.L[2] + 1)
                fd, ff_ = np.zeros(cap), np.zeros(cap)
                keep.append((fd, ff_))
                outs[i].displ = fd.ctypes.data_as(C.POINTER(C.c_double))
                outs[i].force = ff_.ctypes.data_as(C.POINTER(C.c_double))
        self._check(self.lib.dtc_solve_batch(self.handle, ins, n, outs))
        return _results(outs, keep if want_fields else None, m2)

    def _macro2(self, outs):
        """Macro order 2: one dtc_macro2_out per record (the 60-load-case leaves)."""
        if self.macro_order != 2:
            return None
        m2 = (capi.Macro2Out * len(outs))()
        for i in range(len(outs)):
            outs[i].macro2 = C.cast(C.byref(m2, i * C.sizeof(capi.Macro2Out)), C.POINTER(capi.Macro2Out))
        return m2

    def solve_device_moduli(self, domains, e_ptrs):
        """solve() with each domain's per-voxel moduli in device memory: e_ptrs[i] is the device
        address of L0*L1*L2 float32 values (x fastest), or 0 for none."""
        n = len(domains)
        ins = (capi.DomainIn * n)(*[d.struct for d in domains])
        outs = (capi.DomainOut * n)()
        m2 = self._macro2(outs)
        ptrs = (C.c_void_p * n)(*[C.c_void_p(int(p)) if p else None for p in e_ptrs])
        self._check(self.lib.dtc_solve_batch_device_moduli(self.handle, ins, n, outs, ptrs))
        return _results(outs, None, m2)

    def energy_grad_device(self, dloss_dc, grad_ptrs):
        """energy_grad() into device memory: grad_ptrs[i] is the device address of the L0*L1*L2
        float32 gradient of domain i."""
        dl = np.ascontiguousarray(np.asarray(dloss_dc, dtype=np.float64).reshape(-1, 6, 6).transpose(0, 2, 1))
        n = dl.shape[0]
        ptrs = (C.c_void_p * n)(*[C.c_void_p(int(p)) for p in grad_ptrs])
        self._check(self.lib.dtc_energy_grad_device(self.handle, dl.ctypes.data_as(C.POINTER(C.c_double)), ptrs, n))

    def mesh_batch(self, domains, macro_order=1):
        """mesh_domain() for many domains of one element type, computed on the device
        (dtc_mesh_batch)."""
        n = len(domains)
        ins = (capi.DomainIn * n)(*[d.struct for d in domains])
        made = [_mesh_out(d, macro_order) for d in domains]
        outs = (capi.MeshOut * n)(*[m[0] for m in made])
        self._check(self.lib.dtc_mesh_batch(self.handle, ins, n, outs))
        return [_mesh_result(d, outs[i], made[i][1]) for i, d in enumerate(domains)]

    def rotation_search(self, ee):
        """CR1/CR2 rotation search of given symmetric 6x6 tensors (n x 6 x 6): result dicts with
        the "cr1" and "cr2" entries of solve()."""
        ee = np.asarray(ee, dtype=np.float64).reshape(-1, 6, 6)
        n = ee.shape[0]
        flat = np.ascontiguousarray(ee.transpose(0, 2, 1))   # column-major per tensor
        outs = (capi.DomainOut * n)()
        self._check(self.lib.dtc_rotation_search(self.handle, flat.ctypes.data_as(C.POINTER(C.c_double)), n, outs))
        return [{k: r[k] for k in ("cr1", "cr2")} for r in _results(outs, None)]

    def stats(self):
        ms, launches, dofit = C.c_double(), C.c_int64(), C.c_double()
        self._check(self.lib.dtc_get_stats(self.handle, C.byref(ms), C.byref(launches), C.byref(dofit)))
        return {"ms_solve": ms.value, "kernel_launches": launches.value, "dof_iterations": dofit.value}

    def kernel_stats(self):
        """Per kernel class: launches, CUDA-event ms, algorithmic bytes/flops per launch."""
        buf = (capi.KernelStats * 32)()
        cnt = C.c_int32()
        self._check(self.lib.dtc_get_kernel_stats(self.handle, buf, 32, C.byref(cnt)))
        return {buf[i].name.decode(): {"launches": buf[i].launches, "ms_total": buf[i].ms_total,
                                       "bytes_per_launch": buf[i].bytes_per_launch,
                                       "flops_per_launch": buf[i].flops_per_launch}
                for i in range(cnt.value)}

    def energy_grad(self, dloss_dc, grads):
        """dL/dE_voxel of the last solve; grads: list of float32 arrays shaped like phi."""
        dl = np.ascontiguousarray(np.asarray(dloss_dc, dtype=np.float64).reshape(-1, 6, 6).transpose(0, 2, 1))
        n = dl.shape[0]
        ptrs = (C.POINTER(C.c_float) * n)(*[g.ctypes.data_as(C.POINTER(C.c_float)) for g in grads])
        self._check(self.lib.dtc_energy_grad(self.handle, dl.ctypes.data_as(C.POINTER(C.c_double)), ptrs, n))


def solve_batch(domains, want_fields=False, **options):
    with Solver(**options) as s:
        return s.solve(domains, want_fields=want_fields)


def element_stiffness(elem_type, E, a, nu):
    """Voxel element stiffness (Hexe08 / Hexe20 of the reference), (3n x 3n) float64."""
    nd = 3 * elem_type
    ke = np.zeros((nd, nd), order="F")
    rc = capi.load().dtc_element_stiffness(elem_type, E, a, nu, ke.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != capi.DTC_OK:
        raise DTCError(rc, "dtc_element_stiffness failed")
    return ke


def _mesh_out(domain, macro_order=1):
    nl = 60 if macro_order == 2 else 24
    L = domain.L
    nen = domain.elem_type
    m = 1 if nen == HEX08 else 2
    max_nodes = (m * L[0] + 1) * (m * L[1] + 1) * (m * L[2] + 1)
    max_elems = L[0] * L[1] * L[2]
    elems = np.zeros(nen * max_elems, np.int64)
    nodes = np.zeros(3 * max_nodes)
    bids = np.zeros(max_nodes, np.int64)
    bvals = np.zeros(nl * 3 * max_nodes)
    o = capi.MeshOut()
    o.macro_order = macro_order
    o.cap_elems, o.cap_nodes = max_elems, max_nodes
    o.elems = elems.ctypes.data_as(C.POINTER(C.c_int64))
    o.nodes = nodes.ctypes.data_as(C.POINTER(C.c_double))
    o.bnode_ids = bids.ctypes.data_as(C.POINTER(C.c_int64))
    o.bnode_vals = bvals.ctypes.data_as(C.POINTER(C.c_double))
    return o, (elems, nodes, bids, bvals)


def _mesh_result(domain, o, keep):
    elems, nodes, bids, bvals = keep
    nl = 60 if o.macro_order == 2 else 24
    nen = domain.elem_type
    ne, nn, nb = o.ne, o.nn, o.nb
    return {"status": o.status, "ne": ne, "nn": nn, "nb": nb, "last_elem_partial": bool(o.last_elem_partial),
            "elems": elems[: nen * ne].reshape(ne, nen), "nodes": nodes[: 3 * nn].reshape(nn, 3),
            "bnode_ids": bids[:nb], "bnode_vals": bvals[: nl * 3 * nb].reshape(nl, 3 * nb, order="F")}


def mesh_domain(domain, macro_order=1):
    """Reference mesh + boundary conditions of one domain (host only, no GPU needed); the
    prescribed values are those of the 24 (macro order 1) or 60 (macro order 2) load cases."""
    lib = capi.load()
    o, keep = _mesh_out(domain, macro_order)
    rc = lib.dtc_mesh_domain(C.byref(domain.struct), C.byref(o))
    if rc != capi.DTC_OK:
        raise DTCError(rc, "dtc_mesh_domain failed")
    return _mesh_result(domain, o, keep)
