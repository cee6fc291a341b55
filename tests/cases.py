"""Shared helpers: golden fixtures and synthetic cases for the tests."""
from __future__ import annotations

import json
import os

import numpy as np

from oracle import dgm_io, ics

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(case):
    z = np.load(os.path.join(GOLDEN, case + ".npz"))
    meta = json.loads(str(z["meta"]))
    mesh = dgm_io.Mesh(int(z["dim"]), z["verts"], z["con"], z["porder"], z["qorder"])
    return mesh, meta, z["modal"]


# boundary kinds of the oracle and of the engine (ora_set_bc / dgmx_set_boundary)
BC_SLIP_WALL, BC_ISOTHERMAL_WALL, BC_STATE, BC_SUBSONIC_OUTFLOW, BC_SUPERSONIC_OUTFLOW = 1, 2, 3, 4, 5


def bc_records(tags, sides, bct, physics):
    """(eid, sid, kind, a, b) records from .bc tags and the .bct database:
    every "*wall*" code is a slip wall for Euler 3-D; for Navier-Stokes 3-D an
    isothermal_wall block {Tw Eref} is the isothermal wall."""
    out = []
    for t, (e, s) in zip(tags, sides):
        code, vals = bct[t]
        if physics == 9:
            assert code == "isothermal_wall", code
            out.append((int(e), int(s), BC_ISOTHERMAL_WALL, float(vals[0]), float(vals[1])))
        else:
            assert "wall" in code, code
            out.append((int(e), int(s), BC_SLIP_WALL, 0.0, 0.0))
    return out


def load_wall_golden(case):
    """A golden case with boundary sides: mesh, meta, final modal state,
    initial modal state and the boundary records."""
    z = np.load(os.path.join(GOLDEN, case + ".npz"))
    meta = json.loads(str(z["meta"]))
    mesh = dgm_io.Mesh(int(z["dim"]), z["verts"], z["con"], z["porder"], z["qorder"])
    rec = bc_records(meta["bc_tags"], z["bc_sides"], meta["bct"], meta["inp"]["eqntype"])
    return mesh, meta, z["modal"], z["ic_modal"], rec


def golden_ic(meta, x, y, z, nf, gamma=1.4):
    code, toks = meta["ic_code"].lower(), meta["ic_tokens"]
    if code == "acousticpulse":
        return ics.acoustic_pulse(x, float(toks[0]), float(toks[1]), float(toks[2]), gamma)
    if code == "vortex":
        nv = int(toks[0])
        vals = [float(t) for t in toks[1:1 + 5 * nv]]
        return ics.vortex_ic(x, y, [vals[5 * i:5 * i + 5] for i in range(nv)], gamma, nf)
    raise ValueError(code)


def diff_norms(U, V, wj):
    """Per-field Linf and L2 of U-V and of V (Domain::diff, src/Domain.cpp:1000-1066)."""
    out = []
    area = wj.sum()
    for n in range(U.shape[0]):
        d = U[n] - V[n]
        out.append(dict(linf=np.abs(d).max(), l2=np.sqrt((d * d * wj).sum() / area),
                        ref_linf=np.abs(V[n]).max(), ref_l2=np.sqrt((V[n] ** 2 * wj).sum() / area)))
    return out


def passes_dgm_diff(norms, aeps, reps, repsM=float(np.sqrt(np.finfo(float).eps))):
    """dgm_diff pass/fail: absolute test on Linf/L2, relative test where the
    reference norm is above repsM (src/Domain.cpp:1023-1055)."""
    for f in norms:
        if f["linf"] > aeps or f["l2"] > aeps:
            return False
        if f["ref_linf"] > repsM and f["linf"] / f["ref_linf"] > reps:
            return False
        if f["ref_l2"] > repsM and f["l2"] / f["ref_l2"] > reps:
            return False
    return True


# Face vertex lists (Hex: src/Hex.cpp:68-69; Quad edges: consecutive vertices)
HEX_FACES = [(0, 1, 2, 3), (0, 1, 5, 4), (1, 2, 6, 5), (3, 2, 6, 7), (0, 3, 7, 4), (4, 5, 6, 7)]
QUAD_EDGES = [(0, 1), (1, 2), (3, 2), (0, 3)]


def rotated_box(dim, n, lo, hi, p, q=0, seed=0):
    """Periodic box whose elements have randomly rotated local frames (vertex
    lists cycled about the z axis, and for Hexes optionally turned upside
    down), with the connectivity rebuilt from face centroids.  Exercises the
    side orientation flags (src/Field.cpp:416-680)."""
    base = dgm_io.box_mesh(dim, n, lo, hi, p, q)
    rng = np.random.default_rng(seed)
    verts = base.verts.copy()
    for e in range(base.ne):
        r = int(rng.integers(4))
        if dim == 2:
            order = [(v + r) % 4 for v in range(4)]
        else:
            bot = [(v + r) % 4 for v in range(4)]
            order = bot + [b + 4 for b in bot]
            if rng.integers(2):  # turn upside down: swap bottom/top, keep orientation
                order = [order[4], order[7], order[6], order[5], order[0], order[3], order[2], order[1]]
        verts[e] = base.verts[e][order]
    lo_a = np.broadcast_to(np.asarray(lo, float), (dim,))
    L = np.broadcast_to(np.asarray(hi, float), (dim,)) - lo_a
    faces = HEX_FACES if dim == 3 else QUAD_EDGES
    key = {}
    for e in range(base.ne):
        for f, fv in enumerate(faces):
            c = verts[e][list(fv)][:, :dim].mean(axis=0)
            c = np.mod(c - lo_a + 1e-9 * L, L) - 1e-9 * L
            k = tuple(np.round(c / L * 4 * max(n if hasattr(n, "__len__") else [n]), 6))
            key.setdefault(k, []).append((e, f))
    con = []
    for e in range(base.ne):
        for f, fv in enumerate(faces):
            c = verts[e][list(fv)][:, :dim].mean(axis=0)
            c = np.mod(c - lo_a + 1e-9 * L, L) - 1e-9 * L
            k = tuple(np.round(c / L * 4 * max(n if hasattr(n, "__len__") else [n]), 6))
            pair = [x for x in key[k] if x != (e, f)]
            assert len(pair) == 1, (e, f, key[k])
            con.append([e, f, pair[0][0], pair[0][1]])
    return dgm_io.Mesh(dim, verts, np.array(con, np.int32), base.porder, base.qorder)
