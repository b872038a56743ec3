"""PureDat trees: the reference's on-disk format for CT volumes and results
(f-src/mod_puredat.f90).

A tree is a `<name>.head` text file describing nested branches and leaves, and one raw stream
file per data type next to it (`<name>.int1.st`, `.int2.st`, `.int4.st`, `.int8.st`,
`.real8.st`, `.char.st`, `.log.st`; mod_puredat.f90:1364-1370) holding every leaf's values at
its 1-based element range [lower_bound, upper_bound] of that type's stream.  The head lists a
branch (description, counts, stream sizes when the branch owns the streams), then its leaves,
then its sub-branches, depth first (write_branch / write_leaf, mod_puredat.f90:4648-4697).

Reading a domain's voxels follows the reference's block read of the "Scalar data" leaf
(f-src/mod_struct_preprocess.f90:193-242): rows of L0 values at element
vdim0*vdim1*(z-1) + vdim0*(y-1) + (xa0-1) + lbound - 1, for y, z over the domain.  Host code
only; it feeds `Domain` (phi) and `synth.volume_domains`' decomposition.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

# type_of_data -> (stream suffix, numpy dtype); 6 = characters, 7 = Fortran logical(1)
TYPES = {1: ("int1", np.int8), 2: ("int2", "<i2"), 3: ("int4", "<i4"), 4: ("int8", "<i8"), 5: ("real8", "<f8"),
         6: ("char", "S1"), 7: ("log", np.int8)}


@dataclass
class Leaf:
    desc: str
    dat_no: int
    dat_ty: int
    lbound: int
    ubound: int


@dataclass
class Branch:
    desc: str
    leaves: list = field(default_factory=list)
    branches: list = field(default_factory=list)
    streams: list | None = None   # dim_st of the 7 streams when the branch owns them
    log_sep: str = "  "           # separator after <size_log_stream> as written ("  " by write_branch)


def _value(line, tag):
    if not line.startswith(tag):
        raise ValueError(f"PureDat head: expected {tag!r}, got {line!r}")
    return line[len(tag):].strip()


def _desc(line):
    v = _value(line, "<description>")
    if not (len(v) >= 2 and v[0] == "'" and v[-1] == "'"):
        raise ValueError(f"PureDat head: unquoted description {line!r}")
    return v[1:-1]


def read_head(path) -> Branch:
    """Parse a `.head` file into its root branch."""
    lines = Path(path).read_text().splitlines()
    pos = [0]

    def nxt():
        if pos[0] >= len(lines):
            raise ValueError("PureDat head: unexpected end of file")
        line = lines[pos[0]]
        pos[0] += 1
        return line

    def branch():
        if nxt().strip() != "<==branch==>":
            raise ValueError("PureDat head: branch separator expected")
        b = Branch(_desc(nxt()))
        nb = int(_value(nxt(), "<no_of_branches>"))
        nl = int(_value(nxt(), "<no_of_leaves>"))
        if _value(nxt(), "<streams_allocated>") == "T":
            b.streams = []
            for tag in ("int1", "int2", "int4", "int8", "real", "char"):
                b.streams.append(int(_value(nxt(), f"<size_{tag}_stream>")))
            line = nxt()
            rest = line[len("<size_log_stream>"):]
            b.log_sep = rest[: len(rest) - len(rest.lstrip())]
            b.streams.append(int(_value(line, "<size_log_stream>")))
        for _ in range(nl):
            if nxt().strip() != "<--leaf-->":
                raise ValueError("PureDat head: leaf separator expected")
            b.leaves.append(Leaf(_desc(nxt()), int(_value(nxt(), "<no_of_data>")),
                                 int(_value(nxt(), "<type_of_data>")), int(_value(nxt(), "<lower_bound>")),
                                 int(_value(nxt(), "<upper_bound>"))))
        for _ in range(nb):
            b.branches.append(branch())
        return b

    return branch()


def head_text(root: Branch) -> str:
    """The `.head` text of a tree, line for line as write_branch / write_leaf write it."""
    out = []

    def branch(b):
        out.append("<==branch==>")
        out.append(f"<description> '{b.desc}'")
        out.append(f"<no_of_branches> {len(b.branches)}")
        out.append(f"<no_of_leaves> {len(b.leaves)}")
        if b.streams is not None:
            out.append("<streams_allocated> T")
            for tag, v in zip(("int1", "int2", "int4", "int8", "real", "char"), b.streams):
                out.append(f"<size_{tag}_stream> {v}")
            out.append(f"<size_log_stream>{b.log_sep}{b.streams[6]}")
        else:
            out.append("<streams_allocated> F")
        for lf in b.leaves:
            out.extend(["<--leaf-->", f"<description> '{lf.desc}'", f"<no_of_data> {lf.dat_no}",
                        f"<type_of_data> {lf.dat_ty}", f"<lower_bound> {lf.lbound}", f"<upper_bound> {lf.ubound}"])
        for sb in b.branches:
            branch(sb)

    branch(root)
    return "\n".join(out) + "\n"


def write_head(path, root: Branch):
    Path(path).write_text(head_text(root))


class Tree:
    """A tree on disk: `<dir>/<name>.head` and its stream files `<dir>/<name>.<type>.st`."""

    def __init__(self, head_path):
        self.head = Path(head_path)
        if self.head.suffix != ".head":
            raise ValueError("a PureDat tree is named by its .head file")
        self.root = read_head(self.head)
        self.prefix = str(self.head)[: -len(".head")]

    def stream_file(self, dat_ty):
        return f"{self.prefix}.{TYPES[dat_ty][0]}.st"

    def find(self, desc) -> Leaf:
        """First leaf with this description, depth first."""
        def walk(b):
            for lf in b.leaves:
                if lf.desc == desc:
                    return lf
            for sb in b.branches:
                r = walk(sb)
                if r is not None:
                    return r
            return None
        lf = walk(self.root)
        if lf is None:
            raise KeyError(desc)
        return lf

    def leaf_map(self, leaf: Leaf):
        """The leaf's values as a read-only memory map of its stream file."""
        dt = np.dtype(TYPES[leaf.dat_ty][1])
        return np.memmap(self.stream_file(leaf.dat_ty), dtype=dt, mode="r", offset=(leaf.lbound - 1) * dt.itemsize,
                         shape=(leaf.dat_no,))

    def read(self, desc):
        return np.array(self.leaf_map(self.find(desc)))

    def volume_info(self):
        """(vdim, grid spacings) of a scalar data structure."""
        return tuple(int(v) for v in self.read("Number of voxels per direction")), \
            tuple(float(v) for v in self.read("Grid spacings"))

    def read_domain(self, xa_n, L):
        """Voxels of the domain starting at the 1-based voxel xa_n with L voxels per edge, as
        phi[z][y][x] (x fastest): the elements the reference's row reads of the "Scalar data"
        leaf take (mod_struct_preprocess.f90:225-242), through a memory map of the stream."""
        vdim, _ = self.volume_info()
        lf = self.find("Scalar data")
        if lf.dat_no != vdim[0] * vdim[1] * vdim[2]:
            raise ValueError("Scalar data does not hold vdim(1)*vdim(2)*vdim(3) values")
        for d in range(3):
            if xa_n[d] < 1 or xa_n[d] + L[d] - 1 > vdim[d]:
                raise ValueError("domain outside the volume")
        vol = self.leaf_map(lf).reshape(vdim[2], vdim[1], vdim[0])
        x0, y0, z0 = (int(v) - 1 for v in xa_n)
        return np.ascontiguousarray(vol[z0: z0 + L[2], y0: y0 + L[1], x0: x0 + L[0]])


def puredat_domains(head_path, L):
    """The reference's decomposition of a scalar volume into cubic domains of L voxels
    (synth.volume_domains: 1-voxel frame, numbering x fastest), read lazily from the stream:
    yields (domain number, xa_n, phi, grid spacings)."""
    t = Tree(head_path)
    vdim, delta = t.volume_info()
    nd = [(vdim[0] - 2) // L, (vdim[1] - 2) // L, (vdim[2] - 2) // L]
    for k in range(nd[2]):
        for j in range(nd[1]):
            for i in range(nd[0]):
                xa = (L * i + 2, L * j + 2, L * k + 2)
                yield i + j * nd[0] + k * nd[0] * nd[1], xa, t.read_domain(xa, (L, L, L)), delta


def write_scalar_tree(head_path, volume, spacing, origin=(0, 0, 0), shift=(0.0, 0.0, 0.0), content="scalar field",
                      name=None):
    """Write a scalar data structure like the reference's converted CT volumes: leaves
    'Scalar data' (int1/int2/int4 by the volume's dtype), 'Number of voxels per direction',
    'Origin' (int4), 'Grid spacings', 'Origin shift against global coordinate system' (real8),
    'Field content description' (char).  volume[z][y][x]."""
    vol = np.ascontiguousarray(volume)
    ty = {1: 1, 2: 2, 4: 3}.get(vol.dtype.itemsize) if vol.dtype.kind == "i" else None
    if ty is None:
        raise ValueError("scalar data must be int8, int16 or int32")
    vdim = (vol.shape[2], vol.shape[1], vol.shape[0])
    head = Path(head_path)
    prefix = str(head)[: -len(".head")]
    desc = content.encode()
    ints = {}   # stream type -> arrays in stream order
    leaves = []
    pos = {t: 1 for t in TYPES}

    def add(desc_, ty_, arr):
        arr = np.ascontiguousarray(arr, dtype=np.dtype(TYPES[ty_][1])).ravel()
        leaves.append(Leaf(desc_, arr.size, ty_, pos[ty_], pos[ty_] + arr.size - 1))
        pos[ty_] += arr.size
        ints.setdefault(ty_, []).append(arr)

    add("Scalar data", ty, vol)
    add("Number of voxels per direction", 3, np.array(vdim))
    add("Origin", 3, np.array(origin))
    add("Grid spacings", 5, np.array(spacing, dtype=float))
    add("Origin shift against global coordinate system", 5, np.array(shift, dtype=float))
    add("Field content description", 6, np.frombuffer(desc, dtype="S1"))
    root = Branch(name or f"{head.stem} scalar data structure", leaves=leaves,
                  streams=[pos[t] - 1 for t in (1, 2, 3, 4, 5, 6, 7)], log_sep=" ")
    for t, arrs in ints.items():
        with open(f"{prefix}.{TYPES[t][0]}.st", "wb") as f:
            for a in arrs:
                f.write(a.tobytes())
    write_head(head, root)
    return Tree(head)


# The result record of one domain: the 24 leaves of the "Averaged Material Properties" branch
# (f-src_main/dtc.f90:738-777; f-src_main/struct_process.f90:704-741), in order, with their
# type (4 = int8, 5 = real8) and values per domain for the linear macro element (24 load cases).
RESULT_LEAVES = [
    ("Domain number", 4, 1), ("Number of Elements", 4, 1), ("Number of Nodes", 4, 1), ("Collected logs", 4, 24),
    ("Start Time", 5, 1), ("Duration", 5, 1), ("Domain forces", 5, 576), ("Effective numerical stiffness", 5, 576),
    ("Symmetry deviation - effective numerical stiffness", 5, 1), ("Averaged stresses", 5, 144),
    ("Averaged strains", 5, 144), ("Effective stiffness", 5, 36), ("Symmetry deviation - effective stiffness", 5, 1),
    ("Averaged Effective stiffness", 5, 36), ("Symmetry deviation - Averaged effective stiffness", 5, 1),
    ("Rotation Angle CR_1", 5, 1), ("Rotation Vector CR_1", 5, 3), ("Final coordinate system CR_1", 5, 9),
    ("Optimized Effective stiffness CR_1", 5, 36), ("Rotation Angle CR_2", 5, 1), ("Rotation Vector CR_2", 5, 3),
    ("Final coordinate system CR_2", 5, 9), ("Optimized Effective stiffness CR_2", 5, 36),
    ("Effective density", 5, 1)]


def _record_values(r, start_time, duration):
    """The 24 leaf values of one result dict (Solver.solve), matrices flattened column-major
    as the reference's reshape writes them."""
    f = lambda m: np.asarray(m, dtype=float).reshape(-1, order="F")   # noqa: E731
    cr = [r.get("cr1", {}), r.get("cr2", {})]
    out = [[r["domain_number"]], [r["ne"]], [r["nn"]], np.asarray(r["iters"], dtype=np.int64),
           [start_time], [duration], f(r["ff"]), f(r["kmacro"]), [r["sym_k"]],
           np.zeros(144), np.zeros(144), f(r["c"]), [r["sym_c"]], f(r["ee"]), [r["sym_ee"]]]
    for k in cr:
        out += [[k.get("angle", 0.0)], np.asarray(k.get("n", np.zeros(3)), dtype=float),
                f(k.get("aa", np.zeros((3, 3)))), f(k.get("ee", np.zeros((6, 6))))]
    out.append([r["density"]])
    return out


def write_result_tree(head_path, results, *, name=None, start_time=0.0, duration=0.0, decomposition=None):
    """Write the results of a batch (Solver.solve dicts, in domain order) as a PureDat tree with
    the reference's result branch "Averaged Material Properties": its 24 leaves, each holding
    the values of every domain back to back (domain i at offset i * values-per-domain, as the
    reference's workers write them at their comm_nn offsets, f-src_main/struct_process.f90:
    1230-1245), int8 leaves 1-4 in `<name>.int8.st`, real8 leaves 5-24 in `<name>.real8.st`.
    decomposition: optional dict of the 'Global domain decomposition' leaves (x_D, x_D_phy,
    delta, nn_D, ...) written as a branch before the results, like the reference's tree.
    Leaf "Collected logs" holds each load case's CG iteration count (the reference logs its
    24 stage marks there), "Averaged stresses/strains" hold zeros (the reference never computes
    them), "Start Time"/"Duration" the given batch values."""
    head = Path(head_path)
    prefix = str(head)[: -len(".head")]
    pos = {t: 1 for t in TYPES}
    data = {t: [] for t in TYPES}

    def add(desc, ty, arr):
        arr = np.ascontiguousarray(arr, dtype=np.dtype(TYPES[ty][1])).ravel()
        lf = Leaf(desc, arr.size, ty, pos[ty], pos[ty] + arr.size - 1)
        pos[ty] += arr.size
        data[ty].append(arr)
        return lf

    branches = []
    if decomposition:
        dleaves = [add(k, 4 if np.asarray(v).dtype.kind in "iu" else 5, np.atleast_1d(v))
                   for k, v in decomposition.items()]
        branches.append(Branch("Global domain decomposition", leaves=dleaves))
    recs = [_record_values(r, start_time, duration) for r in results]
    leaves = []
    for j, (desc, ty, per) in enumerate(RESULT_LEAVES):
        vals = [np.asarray(rec[j]).ravel() for rec in recs]
        if any(v.size != per for v in vals):
            raise ValueError(f"leaf {desc!r}: expected {per} values per domain")
        leaves.append(add(desc, ty, np.concatenate(vals) if vals else np.zeros(0)))
    branches.append(Branch("Averaged Material Properties", leaves=leaves))
    root = Branch(name or head.stem, branches=branches, streams=[pos[t] - 1 for t in (1, 2, 3, 4, 5, 6, 7)],
                  log_sep=" ")
    for t, arrs in data.items():
        if arrs:
            with open(f"{prefix}.{TYPES[t][0]}.st", "wb") as fh:
                for a in arrs:
                    fh.write(a.tobytes())
    write_head(head, root)
    return Tree(head)


def read_result_tree(head_path):
    """Per-domain records of a tree written by write_result_tree (or a reference result tree
    laid out the same way): a list of dicts leaf description -> values of that domain."""
    t = Tree(head_path)
    res = None
    def walk(b):
        nonlocal res
        if b.desc == "Averaged Material Properties":
            res = b
        for sb in b.branches:
            walk(sb)
    walk(t.root)
    if res is None:
        raise KeyError("no 'Averaged Material Properties' branch")
    per = {d: n for d, _, n in RESULT_LEAVES}
    n = res.leaves[0].dat_no // per[res.leaves[0].desc]
    vals = {lf.desc: np.array(t.leaf_map(lf)).reshape(n, -1) for lf in res.leaves}
    return [{d: v[i] for d, v in vals.items()} for i in range(n)]


__all__ = ["Leaf", "Branch", "Tree", "read_head", "head_text", "write_head", "puredat_domains", "write_scalar_tree",
           "write_result_tree", "read_result_tree", "RESULT_LEAVES", "TYPES"]
