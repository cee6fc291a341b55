"""Order of accuracy in time of the oracle's integrators on a smooth 2-D
Euler vortex (fixed mesh, so the spatial error cancels): LSRK14 and RK4 are
fourth order, TVD-RK3 third.  LSRK14's golden case (runs/LSRK14) uses
Adv-Diff physics, so this convergence test is what pins its coefficients
(src/TimeInt.cpp:1870-1917) for the Euler path.  LSRK14's error constant is
small, so its order is taken over two halvings of the step, away from the
round-off floor."""
import numpy as np
import pytest

import oracle
from oracle import dgm_io, ics


def _run(inttype, dt, T):
    m = dgm_io.box_mesh(2, (8, 8), -5.0, 5.0, 4)
    P = oracle.Problem(m, oracle.EULER2D)
    x, y, _ = P.coords()
    P.set_state(P.project(ics.isentropic_vortex(x, y, beta=1.0, period=(10.0, 10.0))))
    assert P.advance(inttype, dt, int(round(T / dt))) == 0
    return P.state()


@pytest.mark.parametrize("inttype,order,dts", [(14, 4, (0.04, 0.01)), (4, 4, (0.02, 0.01)), (3, 3, (0.02, 0.01))])
def test_temporal_order(inttype, order, dts):
    T = 0.32
    ref = _run(4, 0.00025, T)
    e = [float(np.sqrt(((_run(inttype, dt, T) - ref) ** 2).mean())) for dt in dts]
    observed = np.log2(e[0] / e[1]) / np.log2(dts[0] / dts[1])
    assert abs(observed - order) < 0.35, (e, observed)
