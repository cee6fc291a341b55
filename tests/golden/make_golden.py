"""Extract the reference's own golden regression cases into npz fixtures.

Run in a container that has the reference checkout mounted (argument: the
reference root).  For each case it stores the mesh (vertices, connectivity,
per-element p/q), the .inp parameters, the first initial condition of the .ic
file, the .tst tolerances and the golden restart's modal coefficients
(runs/<case>.ref, decoded with oracle.dgm_io.read_restart).

Cases (all affine, modal Quad/Hex):
  vhex    Euler3d, TVD-RK3, p=10, 8 hexes, 1000 steps   (runs/vhex.tst)
  vquad   Navier-Stokes 2-D (mu=0.02), TVD-RK3, p=10     (runs/vquad.tst)
  vortex  Navier-Stokes 2-D (mu=0), RK4, p=5/10 mixed     (runs/vortex.tst)
  chan    Navier-Stokes 3-D channel (mu=0.01), TVD-RK3, p=3, 512 hexes, 100
          steps, isothermal walls (runs/chan/chan.{bc,bct}), bulk-flow hold
          (runs/chan/chan.chn), restart initial condition runs/chan/chan.ini
          (runs/chan/chan.tst)
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
WALL_CASES = ["chan/chan"]


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
    for case in WALL_CASES:
        root = os.path.join(ref_root, "runs", case)
        name = os.path.basename(case)
        inp = dgm_io.read_inp(root + ".inp")
        mesh = dgm_io.read_case(root, inp["p"], inp.get("q", 0))
        code, toks = dgm_io.parse_ic(root + ".ic")
        nf = {8: 5, 9: 5}[inp["eqntype"]]
        _, ic_fields, _ = dgm_io.read_restart(os.path.join(os.path.dirname(root), toks[0]), nf, mesh.ne)
        header, fields, nmodes = dgm_io.read_restart(root + ".ref", nf, mesh.ne)
        bcs = dgm_io.read_bc(root + ".bc")
        bct = dgm_io.read_bct(root + ".bct")
        aeps, reps = tolerances(root + ".tst")
        np.savez_compressed(
            os.path.join(out_dir, name + ".npz"),
            verts=mesh.verts, con=mesh.con, porder=mesh.porder, qorder=mesh.qorder,
            dim=mesh.dim, modal=np.stack(fields), nmodes=nmodes, ic_modal=np.stack(ic_fields),
            bc_sides=np.array([[e, s_] for _, e, s_ in bcs], dtype=np.int32),
            meta=json.dumps(dict(inp=inp, ic_code=code, ic_tokens=toks, aeps=aeps, reps=reps,
                                 header=header, bc_tags=[t for t, _, _ in bcs], bct=bct,
                                 channel=os.path.exists(root + ".chn"),
                                 source="runs/%s.{inp,msh,con,bc,bct,chn,ic,ini,ref,tst}" % case)))
        print(name, mesh.ne, nf, int(nmodes.sum()), len(bcs))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DGM_REFERENCE_ROOT", "")
    if not root:
        sys.exit("usage: make_golden.py <reference checkout root> (or set DGM_REFERENCE_ROOT)")
    main(root)
