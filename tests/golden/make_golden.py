"""Extract the reference's own golden regression cases into npz fixtures.

Run in a container that has the reference checkout mounted (argument: the
reference root).  For each case it stores the mesh (vertices, connectivity,
per-element p/q), the .inp parameters, the first initial condition of the .ic
file, the .tst tolerances and the golden restart's modal coefficients
(runs/<case>.ref, decoded with oracle.dgm_io.read_restart).

Cases (all affine, periodic, modal Quad/Hex):
  vhex    Euler3d, TVD-RK3, p=10, 8 hexes, 1000 steps   (runs/vhex.tst)
  vquad   Navier-Stokes 2-D (mu=0.02), TVD-RK3, p=10     (runs/vquad.tst)
  vortex  Navier-Stokes 2-D (mu=0), RK4, p=5/10 mixed     (runs/vortex.tst)
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", ".."))
from oracle import dgm_io  # noqa: E402

CASES = ["vhex", "vquad", "vortex"]


def tolerances(tst_path):
    txt = open(tst_path).read()
    aeps = float(re.search(r"^aeps\s*=\s*([0-9.eE+-]+)", txt, re.M).group(1))
    reps = float(re.search(r"^reps\s*=\s*([0-9.eE+-]+)", txt, re.M).group(1))
    return aeps, reps


def main(ref_root):
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for case in CASES:
        root = os.path.join(ref_root, "runs", case)
        inp = dgm_io.read_inp(root + ".inp")
        mesh = dgm_io.read_case(root, inp["p"], inp.get("q", 0))
        code, toks = dgm_io.parse_ic(root + ".ic")
        nf = {1: 4, 2: 4, 8: 5, 9: 5, 30: 3}[inp["eqntype"]]
        header, fields, nmodes = dgm_io.read_restart(root + ".ref", nf, mesh.ne)
        aeps, reps = tolerances(root + ".tst")
        np.savez_compressed(
            os.path.join(out_dir, case + ".npz"),
            verts=mesh.verts, con=mesh.con, porder=mesh.porder, qorder=mesh.qorder,
            dim=mesh.dim, modal=np.stack(fields), nmodes=nmodes,
            meta=json.dumps(dict(inp=inp, ic_code=code, ic_tokens=toks, aeps=aeps, reps=reps,
                                 header=header, source="runs/%s.{inp,msh,con,ord,ic,ref,tst}" % case)))
        print(case, mesh.ne, nf, int(nmodes.sum()))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
