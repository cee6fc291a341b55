"""Pin the CPU oracle against the reference's own golden restart files.

Each case runs the oracle from the case's initial condition for the .inp's
step count and compares the final state with the decoded runs/<case>.ref using
dgm_diff's absolute/relative L2 and Linf tests at the .tst tolerances.
"""
import numpy as np
import pytest

import oracle
from tests.cases import diff_norms, golden_ic, load_golden, passes_dgm_diff


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
