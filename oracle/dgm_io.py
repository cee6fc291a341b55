"""DGM input files and box meshes, restated in Python for the oracle.

Test infrastructure only.  Readers follow the formats the reference parses:
  * root.msh  -- src/Field.cpp:2257-2600 (header line, "ne nsd", then per
                 element a type line and nsd coordinate rows)
  * root.con  -- src/Field.cpp:3478-3540 ("E eid sid leid lsid")
  * root.ord  -- src/Field.cpp:2295-2322 ("eid p q", q=0 means p+2)
  * root.inp  -- key = value pairs (src/Domain.cpp:294)
  * restart   -- src/Domain.cpp:1721-1780 (10-line text header) and
                 src/vField.cpp:1102-1179 (per field: glen, nModes[ne],
                 disp[ne], then the modal coefficients); the golden files were
                 written with 4-byte integer lengths and displacements.
Box meshes follow src/Mesh.cpp (element id = i + nx*(j + ny*k), periodic
links, counter-clockwise vertex order).
"""
from __future__ import annotations

import dataclasses
import re

import json

import numpy as np


@dataclasses.dataclass
class Mesh:
    dim: int
    verts: np.ndarray        # (ne, nv, 3)
    con: np.ndarray          # (ncon, 4): eid, sid, leid, lsid
    porder: np.ndarray       # (ne,)
    qorder: np.ndarray       # (ne,)

    @property
    def ne(self) -> int:
        return int(self.verts.shape[0])


def read_inp(path: str) -> dict:
    out = {}
    for line in open(path):
        line = line.split("#")[0].strip()
        if "=" not in line:
            continue
        k, v = (s.strip() for s in line.split("=", 1))
        try:
            out[k] = int(v)
        except ValueError:
            try:
                out[k] = float(v)
            except ValueError:
                out[k] = v
    return out


def read_msh(path: str):
    lines = open(path).read().splitlines()
    ne, nsd = (int(t) for t in lines[1].split()[:2])
    nv = 4 if nsd == 2 else 8
    verts = np.zeros((ne, nv, 3))
    i = 2
    for e in range(ne):
        i += 1  # element type line
        for c in range(nsd):
            verts[e, :, c] = [float(t) for t in lines[i].split()[:nv]]
            i += 1
    return nsd, verts


def read_con(path: str) -> np.ndarray:
    rows = []
    for line in open(path).read().splitlines()[2:]:
        t = line.split()
        if len(t) >= 5 and t[0] in ("E", "e"):
            rows.append([int(t[1]), int(t[2]), int(t[3]), int(t[4])])
    return np.array(rows, dtype=np.int32)


def read_case(root: str, p: int, q: int = 0) -> Mesh:
    nsd, verts = read_msh(root + ".msh")
    con = read_con(root + ".con")
    ne = verts.shape[0]
    porder = np.full(ne, p, dtype=np.int32)
    qorder = np.full(ne, q if q else p + 2, dtype=np.int32)
    try:
        lines = open(root + ".ord").read().splitlines()[1:]
        for line in lines:
            t = line.split()
            if len(t) >= 3:
                e, pl, ql = int(t[0]), int(t[1]), int(t[2])
                porder[e] = pl
                qorder[e] = ql if ql else pl + 2
    except FileNotFoundError:
        pass
    return Mesh(nsd, verts, con, porder, qorder)


def box_mesh(dim: int, n, lo, hi, p: int, q: int = 0, periodic: bool = True) -> Mesh:
    """Uniform periodic Quad/Hex box (src/Mesh.cpp:472-490 Quad, 3-D analogue)."""
    n = [int(v) for v in (n if hasattr(n, "__len__") else [n] * dim)]
    lo = [float(v) for v in (lo if hasattr(lo, "__len__") else [lo] * dim)]
    hi = [float(v) for v in (hi if hasattr(hi, "__len__") else [hi] * dim)]
    h = [(hi[d] - lo[d]) / n[d] for d in range(dim)]
    if dim == 2:
        nx, ny = n
        ne = nx * ny
        verts = np.zeros((ne, 4, 3))
        con = []
        corner = [(0, 0), (1, 0), (1, 1), (0, 1)]
        for j in range(ny):
            for i in range(nx):
                e = i + j * nx
                for v, (a, b) in enumerate(corner):
                    verts[e, v, 0] = lo[0] + (i + a) * h[0]
                    verts[e, v, 1] = lo[1] + (j + b) * h[1]
                nn = i + ((j + 1) % ny) * nx
                ss = i + ((j - 1) % ny) * nx
                ee = ((i + 1) % nx) + j * nx
                ww = ((i - 1) % nx) + j * nx
                con += [[e, 0, ss, 2], [e, 1, ee, 3], [e, 2, nn, 0], [e, 3, ww, 1]]
    else:
        nx, ny, nz = n
        ne = nx * ny * nz
        verts = np.zeros((ne, 8, 3))
        con = []
        corner = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
                  (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    e = i + nx * (j + ny * k)
                    for v, (a, b, c) in enumerate(corner):
                        verts[e, v, 0] = lo[0] + (i + a) * h[0]
                        verts[e, v, 1] = lo[1] + (j + b) * h[1]
                        verts[e, v, 2] = lo[2] + (k + c) * h[2]
                    idx = lambda ii, jj, kk: (ii % nx) + nx * ((jj % ny) + ny * (kk % nz))
                    # Hex faces: 0 z-, 1 y-, 2 x+, 3 y+, 4 x-, 5 z+ (src/Hex.cpp:68-69)
                    con += [[e, 0, idx(i, j, k - 1), 5], [e, 1, idx(i, j - 1, k), 3],
                            [e, 2, idx(i + 1, j, k), 4], [e, 3, idx(i, j + 1, k), 1],
                            [e, 4, idx(i - 1, j, k), 2], [e, 5, idx(i, j, k + 1), 0]]
    porder = np.full(ne, p, dtype=np.int32)
    qorder = np.full(ne, q if q else p + 2, dtype=np.int32)
    return Mesh(dim, verts, np.array(con, dtype=np.int32), porder, qorder)


def read_bc(path: str):
    """Boundary sides of a DGM .bc file (src/Field.cpp:4469-4490,
    src/Boundary.cpp:25-75): a header line, the count, then one
    `type eid sid` record per side.  Returns [(type, eid, sid)]."""
    lines = open(path).read().splitlines()
    i = 0
    while not lines[i].split() or not lines[i].split()[0].isdigit():
        i += 1
    nbc = int(lines[i].split()[0])
    out = []
    for line in lines[i + 1:]:
        t = line.split()
        if len(t) >= 3:
            out.append((t[0], int(t[1]), int(t[2])))
        if len(out) == nbc:
            break
    return out


def read_bct(path: str) -> dict:
    """BC type database of a DGM .bct file: `Code Tag { values }` blocks
    (src/Navier_Stokes3d.cpp:416-455).  Returns {tag: (code, [values])}."""
    toks = open(path).read().replace("{", " { ").replace("}", " } ").split()
    out, i = {}, 0
    while i + 1 < len(toks):
        code, tag = toks[i], toks[i + 1]
        i += 2
        vals = []
        if i < len(toks) and toks[i] == "{":
            i += 1
            while toks[i] != "}":
                vals.append(float(toks[i]))
                i += 1
            i += 1
        out[tag] = (code.lower(), vals)
    return out


def read_restart(path: str, nfields: int, ne: int, int_bytes: int = 4):
    """Decode a DGM restart file; returns (header lines, list of per-field
    modal arrays concatenated over elements, nModes per element)."""
    raw = open(path, "rb").read()
    pos = 0
    header = []
    if raw[:1] == b"{":
        # JSON header (src/Domain.cpp:1368-1466): the object, then the rest
        # of its closing line; the binary body follows
        depth, instr = 0, False
        for i, c in enumerate(raw):
            if instr:
                instr = c != ord('"')
            elif c == ord('"'):
                instr = True
            elif c == ord("{"):
                depth += 1
            elif c == ord("}"):
                depth -= 1
                if depth == 0:
                    break
        header = json.loads(raw[:i + 1].decode("latin-1"))
        pos = raw.index(b"\n", i) + 1
    else:
        for _ in range(10):
            nl = raw.index(b"\n", pos)
            header.append(raw[pos:nl].decode("latin-1"))
            pos = nl + 1
    idt = np.int32 if int_bytes == 4 else np.int64
    fields = []
    nmodes = None
    for _ in range(nfields):
        glen = int(np.frombuffer(raw, idt, 1, pos)[0]); pos += int_bytes
        nmodes = np.frombuffer(raw, np.int32, ne, pos).copy(); pos += 4 * ne
        pos += int_bytes * ne  # displacements
        data = np.frombuffer(raw, np.float64, int(nmodes.sum()), pos).copy()
        pos += 8 * int(nmodes.sum())
        assert glen == nmodes.sum(), (glen, nmodes.sum())
        fields.append(data)
    assert pos == len(raw), (pos, len(raw))
    return header, fields, nmodes


def parse_ic(path: str):
    """First initial condition block of a DGM .ic file: (code, tokens)."""
    lines = open(path).read().splitlines()
    code = lines[1].split()[0]
    toks = []
    for line in lines[2:]:
        if not line.strip():
            break
        toks += line.split()
    return code, toks
