"""Generate the golden fixtures under tests/golden/ from the reference's own source text.

The reference (Fortran 90 + PETSc) cannot be compiled or run here, so the only numeric
ground truth it ships is tabulated in its source files.  This script parses those tables
and evaluates them, writing small .npy/.json fixtures that the CPU test-suite compares the
oracle (and the library's host code) against.  It is run once in a container that has the
reference checkout; the fixtures are committed so nothing at test time reads the reference.

Fixtures written:
  ke08_table_nu{NU}.npy   mod_linfe.f90:161-776  Hexe08 C_FE(24,24) table before `* factor`
                          (factor = E*a/(144*(2nu^2+nu-1)), mod_linfe.f90:182)
  ke20_table_nu{NU}.npy   mod_linfe.f90:890-4509 Hexe20 C_FE(60,60) table before `* factor`
                          (factor = E*a*2nu/(256*(2nu^2+nu-1)*2nu), mod_linfe.f90:904)
  uu_hexe8_eps1e-6.npy    mod_write_deck.f90:63-116 init_displ_hexe8, uu(8,3,24)
  vv_lin_eps1e-6.npy      mod_struct_calcmat.f90:1684-1770 init_loadcase_el_order_lin, vv(24,24)
  golden_meta.json        the source line ranges and the evaluation parameters

Usage:  python tests/golden/make_golden.py /path/to/reference-checkout
"""
import json
import re
import sys
from pathlib import Path

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py /path/to/reference-checkout")
REF = Path(sys.argv[1])
OUT = Path(__file__).resolve().parent


def _fortran_expr(expr: str) -> str:
    expr = expr.replace("_rk", "").replace("_8", "")
    expr = re.sub(r"(\d)\.(?!\d)", r"\1.0", expr)  # "0." -> "0.0"
    expr = expr.replace("**", "^^").replace("^^", "**")
    return expr


def ke_table(lines, lo, hi, n, nu):
    K = np.full((n, n), np.nan)
    pat = re.compile(r"^\s*C_FE\((\d+),(\d+)\)\s*=\s*(.+?)\s*$")
    for ln in lines[lo - 1:hi]:
        m = pat.match(ln)
        if m:
            K[int(m.group(1)) - 1, int(m.group(2)) - 1] = eval(_fortran_expr(m.group(3)), {"nu": nu})
    assert np.isfinite(K).all(), "table not completely filled"
    return K


def joined_statements(lines, lo, hi):
    """Join Fortran free-form continuation lines ('&' at end) into statements."""
    out, cur = [], ""
    for ln in lines[lo - 1:hi]:
        s = ln.split("!")[0].rstrip()
        if s.endswith("&"):
            cur += s[:-1] + " "
            continue
        s = s.lstrip()
        if s.startswith("&"):
            s = s[1:]
        cur += s
        out.append(cur)
        cur = ""
    return out


def uu_hexe8(lines, eps):
    uu = np.zeros((8, 3, 24))
    pat = re.compile(r"uu\(:,\s*(\d+),\s*(\d+)\)\s*=\s*\[(.*)\]")
    for st in joined_statements(lines, 63, 116):
        m = pat.search(st)
        if m:
            vals = [eval(_fortran_expr(v.strip()), {"eps": eps}) for v in m.group(3).split(",")]
            assert len(vals) == 8
            uu[:, int(m.group(1)) - 1, int(m.group(2)) - 1] = vals
    return uu


def vv_lin(lines, eps):
    vv = np.zeros((24, 24))
    pat = re.compile(r"vv\(\s*(\d+),:\)\s*=\s*\[(.*)\]")
    env = {"eps": eps, "eps2": 2 * eps, "eps3": 3 * eps, "eps4": 4 * eps}
    n = 0
    for st in joined_statements(lines, 1684, 1770):
        m = pat.search(st)
        if m:
            vals = [eval(_fortran_expr(v.strip()), env) for v in m.group(2).split(",")]
            assert len(vals) == 24
            vv[int(m.group(1)) - 1, :] = vals
            n += 1
    assert n == 24
    return vv


_REAL_LIT = re.compile(r"(?<![\w.])(\d+\.\d*|\.\d+)(_rk)?")


def _fortran_kind_expr(expr: str) -> str:
    """Like _fortran_expr, but a real literal without a kind suffix is a default (single
    precision) REAL in Fortran: `.9*eps` multiplies eps by 0.9 rounded to float32."""
    def lit(m):
        return m.group(1) if m.group(2) else f"f32({m.group(1)})"
    return _REAL_LIT.sub(lit, expr).replace("**", "^^").replace("^^", "**")


def f32(x):
    return float(np.float32(x))


def uu_hexe20(lines, eps):
    """init_displ_hexe20 (mod_write_deck.f90:118-279): uu(20,3,60); its index shift ish = 1
    makes `uu(:,ish+c,ish+m)` component c+1 of load case m+1."""
    uu = np.zeros((20, 3, 60))
    pat = re.compile(r"uu\(:,\s*ish\+(\d+),\s*ish\+(\d+)\)\s*=\s*\[(.*)\]")
    n = 0
    for st in joined_statements(lines, 118, 279):
        m = pat.search(st)
        if m:
            vals = [eval(_fortran_kind_expr(v.strip()), {"eps": eps, "z": 0.0, "f32": f32})
                    for v in m.group(3).split(",")]
            assert len(vals) == 20
            uu[:, int(m.group(1)), int(m.group(2))] = vals
            n += 1
    assert n == 75
    return uu


def vv_quad(lines, e):
    """init_loadcase_el_order_quad (mod_struct_calcmat.f90:1780-2028) as its statements read.

    Returns (table, statements): `table` is what the Fortran assignments leave in vv(60,60)
    (vv = 0, then every `vv(r,:) = [...]` in source order, later ones overwriting earlier
    ones; a statement with more than 60 values keeps its first 60), and `statements` lists
    (source line, row label, values as written) for every statement, so the defects of the
    table can be checked one by one."""
    table = np.zeros((60, 60))
    pat = re.compile(r"vv\(\s*(\d+),:\)\s*=\s*\[(.*)\]")
    stmts = []
    for st in joined_statements(lines, 1780, 2028):
        m = pat.search(st)
        if m:
            raw = [v.strip() for v in m.group(2).split(",")]
            vals = [eval(_fortran_kind_expr(v).replace("- ", "-"), {"e": e, "z": 0.0, "f32": f32}) for v in raw]
            stmts.append((int(m.group(1)), vals))
            table[int(m.group(1)) - 1, :] = vals[:60]
    assert len(stmts) == 60
    return table, stmts


def main():
    linfe = (REF / "f-src/mod_linfe.f90").read_text().splitlines()
    deck = (REF / "f-src/mod_write_deck.f90").read_text().splitlines()
    calc = (REF / "f-src/mod_struct_calcmat.f90").read_text().splitlines()
    meta = {"reference_files": {
        "ke08": "f-src/mod_linfe.f90:161-776", "ke20": "f-src/mod_linfe.f90:890-4509",
        "uu": "f-src/mod_write_deck.f90:63-116", "vv": "f-src/mod_struct_calcmat.f90:1684-1770",
        "uu20": "f-src/mod_write_deck.f90:118-279", "vv_quad": "f-src/mod_struct_calcmat.f90:1780-2028"},
        "nu": [0.3, 0.25], "eps": 1e-6}
    for nu in meta["nu"]:
        np.save(OUT / f"ke08_table_nu{nu}.npy", ke_table(linfe, 161, 776, 24, nu))
        np.save(OUT / f"ke20_table_nu{nu}.npy", ke_table(linfe, 890, 4509, 60, nu))
    np.save(OUT / "uu_hexe8_eps1e-6.npy", uu_hexe8(deck, 1e-6))
    np.save(OUT / "vv_lin_eps1e-6.npy", vv_lin(calc, 1e-6))
    np.save(OUT / "uu_hexe20_eps1e-6.npy", uu_hexe20(deck, 1e-6))
    table, stmts = vv_quad(calc, 1e-6)
    np.save(OUT / "vv_quad_table_eps1e-6.npy", table)
    # every statement as written: row label, value count, values (padded to 61)
    st = np.zeros((len(stmts), 61))
    st_len = np.array([len(v) for _, v in stmts])
    for i, (_, v) in enumerate(stmts):
        st[i, :len(v)] = v
    np.savez(OUT / "vv_quad_statements_eps1e-6.npz", labels=np.array([r for r, _ in stmts]), nvals=st_len,
             values=st)
    (OUT / "golden_meta.json").write_text(json.dumps(meta, indent=1) + "\n")
    print("fixtures written to", OUT)


if __name__ == "__main__":
    main()
