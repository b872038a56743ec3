"""Copies PureDat head files shipped with the reference (a converted CT scalar volume and the
results tree of the solid-cube regression case) into tests/golden/puredat/: the parser and the
writer of m-dtc-direct-tensor-computation_b200/puredat.py are pinned on them byte for byte.
Run from the repository root: python tests/golden/make_puredat_fixtures.py /path/to/reference"""
import shutil
import sys
from pathlib import Path

SRC = [
    "datasets/isotropic_testcase_converted/SC00-0_tc_Dev_BinDecomp_isotropic-HEX08.head",
    "regression/solid_cube/solid_cube_Hex08/solid_cube_Hex08.head",
    "datasets/isotropic_testcase_converted/SC00-0_tc_Pro_DDTC_Tensors/SC00-0_tc_Pro_DDTC_Tensors.head",
]

if __name__ == "__main__":
    ref = Path(sys.argv[1])
    out = Path(__file__).resolve().parent / "puredat"
    out.mkdir(exist_ok=True)
    for s in SRC:
        shutil.copyfile(ref / s, out / Path(s).name)
        print(out / Path(s).name)
