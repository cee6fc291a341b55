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
