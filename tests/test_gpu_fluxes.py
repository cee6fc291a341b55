"""GPU parity of the flux-vector splittings of Euler::convective_flux
(src/Euler.cpp:577-680): Steger-Warming and van Leer on Euler and
Navier-Stokes 2-D, against the oracle's restatement, on straight and
rotated meshes; and the refusals where the reference has no such flux."""
import numpy as np
import pytest

import oracle
from oracle import dgm_io, ics

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


CASES = [
    # name, physics, flux, p, inttype, vis, rotated
    ("euler2d-sw-lsrk14", 1, "stegerwarming", 4, 14, 0.0, False),
    ("euler2d-vl-lsrk14", 1, "vanleer", 4, 14, 0.0, False),
    ("euler2d-sw-rotated-tvd3", 1, "stegerwarming", 3, 3, 0.0, True),
    ("euler2d-vl-rotated-rk4", 1, "vanleer", 3, 4, 0.0, True),
    ("ns2d-sw-rk4", 2, "stegerwarming", 4, 4, 0.02, False),
    ("ns2d-vl-tvd3", 2, "vanleer", 4, 3, 0.02, False),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_splitting_flux_parity(case):
    import dgm_b200
    from tests.cases import rotated_box
    _, phys, flux, p, inttype, vis, rotated = case
    m = rotated_box(2, (6, 6), -5, 5, p, 0, seed=3) if rotated else dgm_b200.meshgen.box(2, (6, 6), -5, 5, p)
    P = oracle.Problem(dgm_io.Mesh(2, m.verts, m.con, m.porder, m.qorder), phys, flux=flux, vis=vis)
    D = dgm_b200.Domain(m, phys, flux=flux, inttype=inttype, vis=vis)
    x, y, _ = P.coords()
    f = ics.vortex_ic(x, y, [(0.0, 0.0, 1.0, 1.0, 0.5)], nf=4)
    f[1] += 0.3 * f[0]   # a mean flow, so faces see both signs of the normal velocity
    f[3] += 0.5 * 0.09 * f[0]
    U0 = P.project(f)
    F_g, F_o = D.time_derivative(U0), P.rhs(U0)
    assert np.linalg.norm(F_g - F_o) <= 1e-12 * np.linalg.norm(U0)
    D_lf = dgm_b200.Domain(m, phys, flux="laxfriedrichs", inttype=inttype, vis=vis)
    assert not np.allclose(F_g, D_lf.time_derivative(U0))   # a different flux ran
    D_lf.close()
    P.set_state(U0)
    D.set_state(f)
    assert P.advance(inttype, 0.005, 10) == 0
    D.advance(0.005, 10)
    assert rel(D.state(), P.state()) < 1e-12
    D.close()


@pytest.mark.parametrize("flux", ["stegerwarming", "vanleer"])
def test_splitting_flux_refusals(flux):
    import dgm_b200
    m3 = dgm_b200.meshgen.box(3, (2, 2, 2), 0, 1, 2)
    with pytest.raises(dgm_b200.DgmxError):
        dgm_b200.Domain(m3, dgm_b200.EULER3D, flux=flux)
    m2 = dgm_b200.meshgen.box(2, (2, 2), 0, 1, 2)
    with pytest.raises(dgm_b200.DgmxError):
        dgm_b200.Domain(m2, dgm_b200.EULER2D, flux=flux, precision=dgm_b200.MIXED)
    with pytest.raises(dgm_b200.DgmxError):
        dgm_b200.Domain(m2, dgm_b200.SHALLOW, flux=flux)
