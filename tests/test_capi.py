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
               "dtc_domain_out": dtc.capi.DomainOut, "dtc_mesh_out": dtc.capi.MeshOut}
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
