"""The oracle's source term (CPU): F -= S at the GLL points before the
projection equals the plain right-hand side minus the projection of S
(projection is linear), for the 2-D physics; 3-D applies none."""
import numpy as np

import oracle
from oracle import dgm_io, ics


def _mesh(dim, n, lo, hi, p):
    import dgm_b200
    m = dgm_b200.meshgen.box(dim, n, lo, hi, p)
    return dgm_io.Mesh(dim, m.verts, m.con, m.porder, m.qorder)


def test_source_is_subtracted_before_projection():
    P = oracle.Problem(_mesh(2, (3, 3), -5, 5, 3), oracle.EULER2D)
    x, y, _ = P.coords()
    U0 = P.project(ics.vortex_ic(x, y, [(0.0, 0.0, 1.0, 1.0, 0.5)], nf=4))
    S = np.stack([np.exp(-(x - k) ** 2 - y ** 2) for k in range(4)])
    F0 = P.rhs(U0)
    P.set_source(S)
    F1 = P.rhs(U0)
    assert np.abs(F1 - (F0 - P.project(S))).max() < 1e-12
    P.set_source(None)
    assert np.array_equal(P.rhs(U0), F0)


def test_no_source_in_3d():
    P = oracle.Problem(_mesh(3, (2, 2, 2), 0, 1, 2), oracle.EULER3D)
    x, y, z = P.coords()
    U0 = P.project(ics.taylor_green(x, y, z, Ma=0.1))
    F0 = P.rhs(U0)
    P.set_source(np.ones((5, x.size)))
    assert np.array_equal(P.rhs(U0), F0)


def test_oracle_time_follows_the_integrators():
    """Domain::t after n steps is n dt for LSRK14, TVD3 and RK4, and a source
    pulse far from the run's times leaves the source off."""
    P = oracle.Problem(_mesh(2, (3, 3), -2, 2, 2), oracle.SHALLOW)
    P.set_sw_balance(False)
    x, y, _ = P.coords()
    U0 = P.project(ics.gaussian_bump(x, y, a=0.3, w=0.5))
    for inttype in (14, 3, 4):
        P.set_time(0.0)
        P.set_state(U0)
        assert P.advance(inttype, 0.001, 7) == 0
        assert abs(P.time() - 0.007) < 1e-15
    F0 = P.rhs(U0)
    P.set_source(np.ones((3, x.size)))
    P.set_source_pulse(100.0, 0.01)
    P.set_time(0.0)
    assert np.array_equal(P.rhs(U0), F0)
