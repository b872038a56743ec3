"""The C-ABI library: loads, exports every symbol include/dtc.h declares, validates inputs."""
import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    text = (ROOT / "include" / "dtc.h").read_text()
    return sorted(set(re.findall(r"\b(dtc_[a-z_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(dtc):
    lib = dtc.capi.load()
    syms = declared_symbols()
    assert "dtc_solve_batch" in syms and "dtc_mesh_domain" in syms
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(dtc.capi.SIGNATURES)
    assert lib.dtc_abi_version() == dtc.capi.ABI_VERSION


def test_default_options_are_the_reference_petsc_options(dtc):
    lib = dtc.capi.load()
    o = dtc.capi.Options()
    lib.dtc_default_options(C.byref(o))
    assert o.rtol == 1e-3 and o.max_it == 500000      # f-src/mod_parameters.f90:31-32
    assert o.precision == dtc.PREC_FP64 and o.abi_version == dtc.capi.ABI_VERSION


def test_struct_layouts_match_the_header(dtc, tmp_path):
    """ctypes mirrors of the C structs have the size and field offsets the C compiler gives."""
    import subprocess
    structs = {"dtc_options": dtc.capi.Options, "dtc_domain_in": dtc.capi.DomainIn,
               "dtc_domain_out": dtc.capi.DomainOut, "dtc_mesh_out": dtc.capi.MeshOut,
               "dtc_macro2_out": dtc.capi.Macro2Out}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dtc.h"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, (cname, f)


def test_mesh_domain_validation(dtc):
    lib = dtc.capi.load()
    d = dtc.Domain(np.ones((3, 3, 3), np.int16))
    out = dtc.capi.MeshOut()
    bad = dtc.capi.DomainIn.from_buffer_copy(d.struct)
    bad.elem_type = 9
    assert lib.dtc_mesh_domain(C.byref(bad), C.byref(out)) == dtc.capi.DTC_ERR_INVALID_ARGUMENT
    bad = dtc.capi.DomainIn.from_buffer_copy(d.struct)
    bad.phi = None
    assert lib.dtc_mesh_domain(C.byref(bad), C.byref(out)) == dtc.capi.DTC_ERR_INVALID_ARGUMENT
    bad = dtc.capi.DomainIn.from_buffer_copy(d.struct)
    bad.delta[1] = 0.06                           # non-cubic voxels (mod_linfe.f90:177-180)
    assert lib.dtc_mesh_domain(C.byref(bad), C.byref(out)) == dtc.capi.DTC_ERR_INVALID_ARGUMENT
    assert lib.dtc_mesh_domain(None, C.byref(out)) == dtc.capi.DTC_ERR_INVALID_ARGUMENT
    assert lib.dtc_element_stiffness(7, 1.0, 1.0, 0.3, None) == dtc.capi.DTC_ERR_INVALID_ARGUMENT


def test_create_reports_missing_device_or_abi(dtc):
    import torch
    lib = dtc.capi.load()
    o = dtc.capi.Options()
    lib.dtc_default_options(C.byref(o))
    o.abi_version = 99
    h = C.c_void_p()
    assert lib.dtc_create(C.byref(h), C.byref(o)) == dtc.capi.DTC_ERR_ABI_MISMATCH
    if not torch.cuda.is_available():
        o.abi_version = dtc.capi.ABI_VERSION
        assert lib.dtc_create(C.byref(h), C.byref(o)) == dtc.capi.DTC_ERR_NO_DEVICE
        with pytest.raises(dtc.DTCError):
            dtc.Solver()


def test_macro_order_option_validation(dtc):
    """Macro order 1 or 2, and no adjoint for macro order 2: other combinations are refused
    before any device is touched."""
    lib = dtc.capi.load()
    h = C.c_void_p()
    for order, est, keep in ((3, 0, 0), (-1, 0, 0), (2, 0, 1), (2, 1, 1)):
        o = dtc.capi.Options()
        lib.dtc_default_options(C.byref(o))
        o.macro_order, o.tensor_estimator, o.keep_displacements = order, est, keep
        assert lib.dtc_create(C.byref(h), C.byref(o)) == dtc.capi.DTC_ERR_INVALID_ARGUMENT
    out = dtc.capi.MeshOut()
    out.macro_order = 3
    d = dtc.Domain(np.ones((3, 3, 3), np.int16))
    assert lib.dtc_mesh_domain(C.byref(d.struct), C.byref(out)) == dtc.capi.DTC_ERR_INVALID_ARGUMENT


def test_result_records_convert_fieldwise(dtc):
    """The batch conversion of dtc_domain_out records (one numpy view per field) gives what
    element-wise reads of the ctypes records give; 24 x 24 / 6 x 6 / 3 x 3 leaves column-major."""
    import sys
    pkg = sys.modules[dtc.__name__]
    cap = dtc.capi
    dt = cap.numpy_dtype(cap.DomainOut)
    assert dt.itemsize == C.sizeof(cap.DomainOut)
    for name, _ in cap.DomainOut._fields_:
        assert dt.fields[name][1] == getattr(cap.DomainOut, name).offset, name
    n = 7
    outs = (cap.DomainOut * n)()
    rng = np.random.default_rng(2)
    for i in range(n):
        o = outs[i]
        o.status, o.refine_steps, o.domain_number, o.ne, o.nn = -i, i + 1, 100 + i, 1000 * i, 77 + i
        for k in range(576):
            o.ff[k] = rng.standard_normal()
            o.kmacro[k] = rng.standard_normal()
        for k in range(24):
            o.iters[k] = int(rng.integers(0, 1000))
            o.relres[k] = rng.random()
        for k in range(36):
            o.c[k], o.ee[k], o.cr1_ee[k], o.cr2_ee[k] = rng.standard_normal(4)
        for k in range(9):
            o.cr1_aa[k], o.cr2_aa[k] = rng.standard_normal(2)
        for k in range(3):
            o.cr1_n[k], o.cr2_n[k] = rng.standard_normal(2)
        o.density, o.sym_c, o.cr1_angle, o.cr2_crit, o.cr2_iters = rng.random(), rng.random(), 1.5, 2.5, 3 + i
    res = pkg._results(outs, None)
    for i, r in enumerate(res):
        o = outs[i]
        assert (r["status"], r["refine_steps"], r["domain_number"], r["ne"], r["nn"]) == (
            o.status, o.refine_steps, o.domain_number, o.ne, o.nn)
        assert np.array_equal(r["ff"], np.array(o.ff[:]).reshape(24, 24, order="F"))
        assert np.array_equal(r["kmacro"], np.array(o.kmacro[:]).reshape(24, 24, order="F"))
        assert np.array_equal(r["iters"], np.array(o.iters[:])) and r["iters"].dtype == np.int64
        assert np.array_equal(r["relres"], np.array(o.relres[:]))
        for k in ("c", "ee"):
            assert np.array_equal(r[k], np.array(getattr(o, k)[:]).reshape(6, 6, order="F"))
        for k in ("cr1", "cr2"):
            assert np.array_equal(r[k]["ee"], np.array(getattr(o, k + "_ee")[:]).reshape(6, 6, order="F"))
            assert np.array_equal(r[k]["aa"], np.array(getattr(o, k + "_aa")[:]).reshape(3, 3, order="F"))
            assert np.array_equal(r[k]["n"], np.array(getattr(o, k + "_n")[:]))
        assert r["density"] == o.density and r["sym_c"] == o.sym_c
        assert r["cr1"]["angle"] == 1.5 and r["cr2"]["crit"] == 2.5 and r["cr2"]["iters"] == 3 + i
