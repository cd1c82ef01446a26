"""The reference's field file formats, so that the GPU path can load MOONS
restart dumps and write files that MOONS and its post-processing read.

* ``export_primitives`` / ``import_primitives`` -- a grid_field as the
  reference's generated ``export_primitives_grid_field`` /
  ``import_primitives_grid_field`` write and read it
  (code/generated_code/grid_field/grid_field.f90:123-158): Fortran
  list-directed records ``s_f`` (the three extents), a label record, the
  values of ``f`` in column-major order, then the labelled records ``s``
  (the three extents) and ``s_1D`` (the number of points).
* ``export_tecplot_3d`` / ``import_tecplot_3d`` -- the 3-D Tecplot POINT
  files of ``exp_3D_1C/2C/3C`` (code/handwritten/IO/base_export.f90:32-159,
  code/handwritten/grid_field/GF_export_import/GF_export.f90:24-110, headers
  code/handwritten/IO/exp_Tecplot_Header.f90:25-31, zone line
  code/handwritten/IO/exp_Tecplot_Zone.f90:21-34): a TITLE and VARIABLES
  header, then per block a ZONE record and one record per point (x, y, z and
  the components), i fastest, the coordinates of the field's data location
  (nodes or cell centres along each axis), ``pad`` points dropped per side.
* ``export_tecplot_2d`` / ``export_tecplot_1d`` -- a plane or a line of a
  field (``exp_2D_*C`` / ``exp_1D_*C``, base_export.f90:45-70, 95-144,
  161-182; GF_export.f90:116-364, comment records :391-432; headers
  exp_Tecplot_Header.f90; zones exp_Tecplot_Zone.f90:36-55).
* ``export_tecplot_0d`` -- a history (step, value) as the reference writes
  its probes (``exp_Header_0D_1C``, ``exp_Zone_0I``).
* ``import_tecplot`` -- reads any of these (comment records skipped).

Reading follows Fortran list-directed input: every READ starts at a new
record, takes values across as many records as it needs and discards the
rest of its last record; values may be separated by blanks, commas or line
ends, may carry a repeat count (``3*0.0``) and a D exponent (``1.0D-3``).
Writing uses 17 significant digits, so a dump read back is bit-identical.
"""
from __future__ import annotations

import os
from typing import Iterable, List, Sequence, TextIO, Tuple, Union

import numpy as np

PathOrFile = Union[str, os.PathLike, TextIO]


# ---- list-directed records -------------------------------------------------

class _Records:
    """Fortran list-directed READ over a text stream."""

    def __init__(self, text: str):
        self.lines = text.splitlines()
        self.pos = 0

    def skip(self):
        """READ(un,*) with no items: consume one record."""
        if self.pos >= len(self.lines):
            raise ValueError("unexpected end of file")
        self.pos += 1

    def read(self, n: int, kind=float) -> List:
        """READ(un,*) of n values starting at the next record."""
        out: List = []
        while len(out) < n:
            if self.pos >= len(self.lines):
                raise ValueError(f"unexpected end of file ({len(out)} of {n} values read)")
            line = self.lines[self.pos]
            self.pos += 1
            for tok in line.replace(",", " ").split():
                if len(out) >= n:
                    break  # the rest of the record is discarded
                rep = 1
                if "*" in tok:
                    r, tok = tok.split("*", 1)
                    rep = int(r)
                v = kind(tok.replace("D", "E").replace("d", "e")) if kind is float else kind(tok)
                out.extend([v] * min(rep, n - len(out)))
        return out


def _text(src: PathOrFile) -> str:
    if hasattr(src, "read"):
        return src.read()
    with open(src) as f:
        return f.read()


def _fmt(v: float) -> str:
    return f"{v:.17E}"


def _write_values(w: TextIO, vals: Iterable[float], per_line: int = 3):
    buf = []
    for v in vals:
        buf.append(_fmt(float(v)))
        if len(buf) == per_line:
            w.write("   " + "   ".join(buf) + "\n")
            buf = []
    if buf:
        w.write("   " + "   ".join(buf) + "\n")


def _open_w(dst: PathOrFile):
    return (dst, False) if hasattr(dst, "write") else (open(dst, "w"), True)


# ---- grid_field export_primitives / import_primitives -----------------------

def export_primitives(f: np.ndarray, dst: PathOrFile):
    """Write a grid_field (3-D array, Fortran order) as the reference's
    export_primitives_grid_field does."""
    a = np.asarray(f, dtype=np.float64)
    if a.ndim != 3:
        raise ValueError("a grid_field is three-dimensional")
    w, own = _open_w(dst)
    try:
        s = a.shape
        w.write(f" {s[0]:11d} {s[1]:11d} {s[2]:11d}\n")
        if all(x > 0 for x in s):
            w.write(" f     = \n")
            _write_values(w, a.ravel(order="F"))
        w.write(" s     = \n")
        w.write(f" {s[0]:11d} {s[1]:11d} {s[2]:11d}\n")
        w.write(" s_1D  = \n")
        w.write(f" {a.size:11d}\n")
    finally:
        if own:
            w.close()


def import_primitives(src: PathOrFile) -> np.ndarray:
    """Read a grid_field written by export_primitives_grid_field (the
    reference's or ours); returns the array in Fortran order.  The stored
    s / s_1D records are checked against the extents."""
    r = _Records(_text(src))
    s = r.read(3, int)
    if not all(x > 0 for x in s):
        raise ValueError("the dump holds no field values (unallocated grid_field)")
    r.skip()
    vals = r.read(s[0] * s[1] * s[2], float)
    r.skip()
    s2 = r.read(3, int)
    r.skip()
    s1d = r.read(1, int)[0]
    if list(s2) != list(s) or s1d != s[0] * s[1] * s[2]:
        raise ValueError(f"inconsistent dump: s_f {s}, s {s2}, s_1D {s1d}")
    return np.asarray(vals, dtype=np.float64).reshape(s, order="F")


# ---- Tecplot POINT files ----------------------------------------------------

def n_along(dl: int) -> Tuple[bool, bool, bool]:
    """Axes along which a data location lives on nodes (capi CC, FX..FZ,
    EX..EZ, NODE; data_location_extend.f90 semantics)."""
    bits = {0: 0, 1: 1, 2: 2, 3: 4, 4: 6, 5: 5, 6: 3, 7: 7}[int(dl)]
    return (bool(bits & 1), bool(bits & 2), bool(bits & 4))


def location_coords(hn: Sequence[np.ndarray], n_along: Sequence[bool]) -> List[np.ndarray]:
    """Coordinates of a data location (get_coordinates_h_g,
    code/handwritten/grid/grid_extend.f90:335-347): node coordinates hn
    (ghosts included) along the axes where the field lives on nodes, cell
    centres hc = (hn[i] + hn[i+1]) / 2 along the others."""
    out = []
    for h, nd in zip(hn, n_along):
        h = np.asarray(h, dtype=np.float64)
        out.append(h if nd else 0.5 * (h[1:] + h[:-1]))
    return out


_COMP = ("x", "y", "z")


def export_tecplot_3d(dst: PathOrFile, coords: Sequence[np.ndarray], comps: Sequence[np.ndarray], name: str,
                      pad: int = 0, zone: int = 1, header: bool = True, dir: int = 0):
    """One block of exp_3D_1C (one component), exp_3D_3C (three) or
    exp_3D_2C (two: the components other than direction ``dir``).
    ``coords`` are the three coordinate arrays of the field's data location
    (location_coords); ``zone`` is the block number written as the zone
    title; ``header`` writes the TITLE / VARIABLES records (first block)."""
    comps = [np.asarray(c, dtype=np.float64) for c in comps]
    s = comps[0].shape
    if any(c.shape != s for c in comps) or [len(c) for c in coords] != list(s):
        raise ValueError("components and coordinates must share the field's shape")
    w, own = _open_w(dst)
    try:
        if header:
            if len(comps) == 1:
                w.write(' TITLE = "3D Scalar Field"\n')
                w.write(f' VARIABLES = "x","y","z","{name}"\n')
            else:
                w.write(' TITLE = "3D Vector Field"\n')
                if len(comps) == 3:
                    kept = (0, 1, 2)
                elif len(comps) == 2 and dir in (1, 2, 3):
                    kept = tuple(d for d in range(3) if d != dir - 1)
                else:
                    raise ValueError("two components need dir (the direction left out), 1..3")
                names = ",".join(f'"{name}_{_COMP[i]}"' for i in kept)
                w.write(f' VARIABLES = "x","y","z",{names}\n')
        I, J, K = (s[0] - 2 * pad, s[1] - 2 * pad, s[2] - 2 * pad)
        w.write(f' ZONE , T ="{zone}", I ={I}, J ={J}, K ={K} DATAPACKING = POINT\n')
        hx, hy, hz = coords
        for k in range(pad, s[2] - pad):
            for j in range(pad, s[1] - pad):
                for i in range(pad, s[0] - pad):
                    row = [hx[i], hy[j], hz[k]] + [c[i, j, k] for c in comps]
                    w.write("   " + "   ".join(_fmt(v) for v in row) + "\n")
    finally:
        if own:
            w.close()


def import_tecplot_3d(src: PathOrFile) -> List[Tuple[Tuple[int, int, int], np.ndarray]]:
    """Read the zones of a 3-D POINT file: a list of ((I, J, K), data) with
    data[i, j, k, v] over the VARIABLES (coordinates first)."""
    lines = _text(src).splitlines()
    nvar = None
    zones = []
    p = 0
    while p < len(lines):
        ln = lines[p].strip()
        p += 1
        if ln.upper().startswith("VARIABLES"):
            nvar = ln.count('"') // 2
        elif ln.upper().startswith("ZONE"):
            toks = ln.replace(",", " ").replace("=", " = ").split()
            kv = {}
            for t_i, t in enumerate(toks):
                if t.upper() in ("I", "J", "K") and t_i + 2 < len(toks) and toks[t_i + 1] == "=":
                    kv[t.upper()] = toks[t_i + 2]
            I, J, K = int(kv["I"]), int(kv["J"]), int(kv["K"])
            if nvar is None:
                raise ValueError("ZONE before VARIABLES")
            r = _Records("\n".join(lines[p:]))
            vals = r.read(I * J * K * nvar, float)
            p += r.pos
            d = np.asarray(vals, dtype=np.float64).reshape(K, J, I, nvar).transpose(2, 1, 0, 3)
            zones.append(((I, J, K), d))
    return zones


_XYZ = ("x", "y", "z")


def _adj(d: int) -> Tuple[int, int]:
    """adj_dir_given_dir: the two other directions (1-based), ascending."""
    return {1: (2, 3), 2: (1, 3), 3: (1, 2)}[d]


def _cp2str(v: float) -> str:
    """cp2str: F40.20, blanks trimmed."""
    return f"{float(v):.20f}"


def _check_dir(dir: int):
    if dir not in (1, 2, 3):
        raise ValueError("dir must be 1, 2 or 3")


def i_midplane(n_cells_with_ghosts: int) -> int:
    """coordinates%i_midplane = sc/2 + 1 (1-based)."""
    return n_cells_with_ghosts // 2 + 1


def export_tecplot_2d(dst: PathOrFile, coords: Sequence[np.ndarray], comps: Sequence[np.ndarray], name: str,
                      dir: int, plane: int, pad: int = 0, zone: int = 1, header: bool = True):
    """One block of exp_2D_1C/2C/3C: the plane of 1-based index ``plane``
    normal to direction ``dir`` (1..3).  ``coords`` are the field's data
    location coordinates (location_coords); with two components they are
    the ones other than ``dir``, as in the reference.  Records: the two
    in-plane coordinates and the components, the first in-plane direction
    fastest."""
    _check_dir(dir)
    comps = [np.asarray(c, dtype=np.float64) for c in comps]
    s = comps[0].shape
    if any(c.shape != s for c in comps) or [len(c) for c in coords] != list(s):
        raise ValueError("components and coordinates must share the field's shape")
    if not 1 <= plane <= s[dir - 1]:
        raise ValueError(f"plane {plane} outside 1..{s[dir - 1]}")
    d1, d2 = _adj(dir)
    nc = len(comps)
    w, own = _open_w(dst)
    try:
        if header:
            if nc == 1:
                w.write(' TITLE = "2D Scalar Field"\n')
                # the reference names the scalar with the normal's suffix
                w.write(f' VARIABLES = "{_XYZ[d1 - 1]}","{_XYZ[d2 - 1]}","{name}_{_XYZ[dir - 1]}"\n')
            else:
                w.write(' TITLE = "2D Vector Field"\n')
                kept = (0, 1, 2) if nc == 3 else (d1 - 1, d2 - 1)
                if nc not in (2, 3):
                    raise ValueError("one, two or three components")
                names = ",".join(f'"{name}_{_XYZ[i]}"' for i in kept)
                w.write(f' VARIABLES = "{_XYZ[d1 - 1]}","{_XYZ[d2 - 1]}",{names}\n')
        w.write(f' ZONE , T ="{zone}", I ={s[d1 - 1] - 2 * pad}, J ={s[d2 - 1] - 2 * pad} DATAPACKING = POINT\n')
        c = _XYZ[dir - 1]
        w.write(f"# Plane direction = {dir}\n")
        w.write(f"# Plane index({c})  = {plane}\n")
        w.write(f"# Plane location({c})  = {_cp2str(coords[dir - 1][plane - 1])}\n")
        for j in range(pad, s[d2 - 1] - pad):
            for i in range(pad, s[d1 - 1] - pad):
                idx = [0, 0, 0]
                idx[dir - 1] = plane - 1
                idx[d1 - 1] = i
                idx[d2 - 1] = j
                row = [coords[d1 - 1][i], coords[d2 - 1][j]] + [a[tuple(idx)] for a in comps]
                w.write("   " + "   ".join(_fmt(v) for v in row) + "\n")
    finally:
        if own:
            w.close()


def export_tecplot_1d(dst: PathOrFile, coords: Sequence[np.ndarray], comps: Sequence[np.ndarray], name: str,
                      dir: int, line: Sequence[int], pad: int = 0, zone: int = 1, header: bool = True):
    """One block of exp_1D_1C/2C/3C: the line along direction ``dir`` through
    the 1-based indices ``line`` of the two other directions (ascending).
    With two components they are the ones other than ``dir``."""
    _check_dir(dir)
    comps = [np.asarray(c, dtype=np.float64) for c in comps]
    s = comps[0].shape
    if any(c.shape != s for c in comps) or [len(c) for c in coords] != list(s):
        raise ValueError("components and coordinates must share the field's shape")
    d1, d2 = _adj(dir)
    if not (1 <= line[0] <= s[d1 - 1] and 1 <= line[1] <= s[d2 - 1]):
        raise ValueError("line indices outside the field")
    nc = len(comps)
    w, own = _open_w(dst)
    try:
        if header:
            if nc == 1:
                w.write(' TITLE = "1D Scalar Field"\n')
                w.write(f' VARIABLES = "{_XYZ[dir - 1]}","{name}"\n')
            else:
                if nc not in (2, 3):
                    raise ValueError("one, two or three components")
                w.write(' TITLE = "1D Vector Field"\n')
                kept = (0, 1, 2) if nc == 3 else (d1 - 1, d2 - 1)
                names = ",".join(f'"{name}_{_XYZ[i]}"' for i in kept)
                w.write(f' VARIABLES = "{_XYZ[dir - 1]}",{names}\n')
        w.write(f' ZONE , T ="{zone}", I ={s[dir - 1] - 2 * pad} DATAPACKING = POINT\n')
        c1, c2 = _XYZ[d1 - 1], _XYZ[d2 - 1]
        w.write(f"# Line direction = {dir}\n")
        w.write(f"# Line index({c1})  = {line[0]}\n")
        w.write(f"# Line index({c2})  = {line[1]}\n")
        w.write(f"# Line location({c1})  = {_cp2str(coords[d1 - 1][line[0] - 1])}\n")
        w.write(f"# Line location({c2})  = {_cp2str(coords[d2 - 1][line[1] - 1])}\n")
        for i in range(pad, s[dir - 1] - pad):
            idx = [0, 0, 0]
            idx[dir - 1] = i
            idx[d1 - 1] = line[0] - 1
            idx[d2 - 1] = line[1] - 1
            row = [coords[dir - 1][i]] + [a[tuple(idx)] for a in comps]
            w.write("   " + "   ".join(_fmt(v) for v in row) + "\n")
    finally:
        if own:
            w.close()


def export_tecplot_0d(dst: PathOrFile, n: Sequence[float], values: Sequence[float], name: str):
    """A probe history as the reference writes it: exp_Header_0D_1C
    (TITLE "0D Scalar Field", VARIABLES "N" and the name), the zone record
    of exp_Zone_0I, then one (N, value) record per entry."""
    n = list(n)
    values = list(values)
    if len(n) != len(values):
        raise ValueError("one value per entry")
    w, own = _open_w(dst)
    try:
        w.write(' TITLE = "0D Scalar Field"\n')
        w.write(f' VARIABLES = "N","{name}"\n')
        w.write(" ZONE DATAPACKING = POINT\n")
        for a, b in zip(n, values):
            w.write("   " + _fmt(a) + "   " + _fmt(b) + "\n")
    finally:
        if own:
            w.close()


def import_tecplot(src: PathOrFile):
    """Read a POINT file of any dimension written by the reference or by the
    exporters here.  Returns (variables, zones): the variable names and a list
    of (extents, data) with data[..., v] over the variables, the first extent
    fastest; a zone without I/J/K (the 0-D history) holds every remaining
    record.  Comment records ("#") are skipped."""
    lines = _text(src).splitlines()
    names: List[str] = []
    zones = []
    p = 0
    while p < len(lines):
        ln = lines[p].strip()
        p += 1
        if not ln or ln.startswith("#"):
            continue
        up = ln.upper()
        if up.startswith("TITLE"):
            continue
        if up.startswith("VARIABLES"):
            body = ln.split("=", 1)[1]
            names = [t.strip().strip('"') for t in body.replace(",", " ").split()]
            continue
        if up.startswith("ZONE"):
            if not names:
                raise ValueError("ZONE before VARIABLES")
            toks = ln.replace(",", " ").replace("=", " = ").split()
            ext = {}
            for t_i, t in enumerate(toks):
                if t.upper() in ("I", "J", "K") and t_i + 2 < len(toks) and toks[t_i + 1] == "=":
                    ext[t.upper()] = int(toks[t_i + 2])
            shape = tuple(ext[k] for k in ("I", "J", "K") if k in ext)
            body = [l for l in lines[p:] if l.strip() and not l.strip().startswith("#")
                    and not l.strip().upper().startswith("ZONE")]
            nv = len(names)
            if shape:
                cnt = int(np.prod(shape)) * nv
                r = _Records("\n".join(l for l in lines[p:] if not l.strip().startswith("#")))
                vals = r.read(cnt, float)
                # advance past the records consumed (comment lines do not count)
                used, k = 0, p
                while used < r.pos and k < len(lines):
                    if not lines[k].strip().startswith("#"):
                        used += 1
                    k += 1
                p = k
                data = np.asarray(vals, dtype=np.float64).reshape(tuple(reversed(shape)) + (nv,))
                data = data.transpose(tuple(reversed(range(len(shape)))) + (len(shape),))
            else:
                rows = []
                for l in body:
                    rows.append([float(t.replace("D", "E").replace("d", "e")) for t in l.replace(",", " ").split()])
                p = len(lines)
                data = np.asarray(rows, dtype=np.float64).reshape(-1, nv)
                shape = (data.shape[0],)
            zones.append((shape, data))
    return names, zones


# ---- fields of the library ---------------------------------------------------

def export_field(field, dst: PathOrFile):
    """export_primitives of a library field (capi.Field or an MHD field view)."""
    export_primitives(field.download(), dst)


def import_field(field, src: PathOrFile):
    """Load a reference dump into a library field of the same shape."""
    a = import_primitives(src)
    if tuple(a.shape) != tuple(field.shape):
        raise ValueError(f"dump shape {a.shape} does not match the field's {tuple(field.shape)}")
    field.upload(a)
