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
