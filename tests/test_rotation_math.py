"""The rotation search's sine and cosine (csrc/ddmath.h): correctly rounded on the angles the
search evaluates, so the GPU and the oracle (quad precision, oracle/dtc_oracle.cpp) see the
same values and the argmin indices of the refinement can be compared bit for bit.

Compiles tests/native/sincos_check.cpp with the host compiler (no GPU needed)."""
import shutil
import subprocess

import pytest

from conftest import ROOT

HDR_DIR = ROOT / "m-dtc-direct-tensor-computation_b200" / "csrc"
SRC = ROOT / "tests" / "native" / "sincos_check.cpp"


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs a host C++ compiler")
def test_sincos_correctly_rounded_on_search_angles(tmp_path):
    exe = tmp_path / "sincos_check"
    subprocess.run(["g++", "-O2", "-std=gnu++17", "-ffp-contract=off", f"-I{HDR_DIR}", str(SRC), "-lquadmath",
                    "-o", str(exe)], check=True)
    p = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    n, bad, libm_bad = map(int, p.stdout.split()[-3:])
    assert n > 500_000 and bad == 0
    # the host libm is not correctly rounded everywhere: the reason both sides avoid it
    print(f"{n} angles, libm differs from the nearest double on {libm_bad}")
