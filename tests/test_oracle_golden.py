"""Pin the CPU oracle against the reference's own golden restart files.

Each case runs the oracle from the case's initial condition for the .inp's
step count and compares the final state with the decoded runs/<case>.ref using
dgm_diff's absolute/relative L2 and Linf tests at the .tst tolerances.
"""
import numpy as np
import pytest

import oracle
from tests.cases import diff_norms, golden_ic, load_golden, load_wall_golden, passes_dgm_diff


@pytest.mark.parametrize("case", ["vhex", "vquad", "vortex"])
def test_oracle_matches_reference_golden(case):
    mesh, meta, modal = load_golden(case)
    inp = meta["inp"]
    P = oracle.Problem(mesh, inp["eqntype"], vis=float(inp.get("vis", 0.0)))
    x, y, z = P.coords()
    U0 = P.project(golden_ic(meta, x, y, z, P.nf))
    P.set_state(U0)
    assert P.advance(inp["inttype"], float(inp["dt"]), int(inp["Nt"])) == 0
    U = P.state()
    G = P.backward(modal)
    norms = diff_norms(U, G, P.wj())
    assert passes_dgm_diff(norms, meta["aeps"], meta["reps"]), norms
    # and the restart (modal) coefficients agree directly
    assert np.abs(P.forward(U) - modal).max() < 1e-12


def test_golden_fixture_shapes():
    for case in ["vhex", "vquad", "vortex"]:
        mesh, meta, modal = load_golden(case)
        assert modal.shape[1] == sum((p + 1) ** mesh.dim for p in mesh.porder)


def test_oracle_matches_channel_golden():
    """runs/chan: Navier-Stokes 3-D channel, 512 hexes at p=3, isothermal
    walls, bulk-flow hold, restart initial condition, 100 TVD-RK3 steps; the
    final state passes dgm_diff against chan.ref at the .tst tolerances
    (aeps 5e-10, reps 1e-8)."""
    mesh, meta, modal, ic_modal, rec = load_wall_golden("chan")
    inp = meta["inp"]
    assert meta["channel"] and len(rec) == 128
    P = oracle.Problem(mesh, inp["eqntype"], vis=float(inp["vis"]))
    P.set_bc(rec)
    P.set_hold_bulk(True)
    P.set_state(P.backward(ic_modal))
    assert P.advance(inp["inttype"], float(inp["dt"]), int(inp["Nt"])) == 0
    U = P.state()
    norms = diff_norms(U, P.backward(modal), P.wj())
    assert passes_dgm_diff(norms, meta["aeps"], meta["reps"]), norms
    assert max(f["linf"] for f in norms) < 1e-10


def test_channel_hold_matters():
    """The bulk-flow hold is not a no-op on this case: 20 steps without it
    differ from 20 steps with it by more than the golden tolerance."""
    mesh, meta, modal, ic_modal, rec = load_wall_golden("chan")
    inp = meta["inp"]
    P = oracle.Problem(mesh, inp["eqntype"], vis=float(inp["vis"]))
    P.set_bc(rec)
    P.set_hold_bulk(False)
    P.set_state(P.backward(ic_modal))
    P.advance(inp["inttype"], float(inp["dt"]), 20)
    Q = oracle.Problem(mesh, inp["eqntype"], vis=float(inp["vis"]))
    Q.set_bc(rec)
    Q.set_hold_bulk(True)
    Q.set_state(Q.backward(ic_modal))
    Q.advance(inp["inttype"], float(inp["dt"]), 20)
    d = diff_norms(P.state(), Q.state(), P.wj())
    assert max(f["linf"] for f in d) > 1e-8
