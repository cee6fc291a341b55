"""The 3-D Roe flux has no reference implementation (Euler3d only builds
Lax-Friedrichs, src/Euler3d.cpp:803-805); the oracle and the engine extend
the reference's 2-D Roe (src/Euler.cpp:682-741) to the rotated (n, s, t)
frame of Euler3d::convective_flux.  Pin the extension: a flow with no z
dependence and no z velocity, run in 3-D with Roe, evolves exactly like the
same flow run in 2-D with the reference's Roe flux (the faces normal to z
carry a uniform state and cancel), and under a rotation of the whole box
the flux turns with it."""
import numpy as np
import pytest

import oracle
from oracle import dgm_io, ics


def _by_element_xy(P2, m2, P3, m3, U2, U3, nx, ny):
    x2, y2, _ = P2.coords()
    x3, y3, z3 = P3.coords()
    q2 = len(x2) // m2.ne
    q3 = len(x3) // m3.ne
    worst = 0.0
    for k in range(m3.ne // (nx * ny)):
        for j in range(ny):
            for i in range(nx):
                e2, e3 = i + nx * j, i + nx * (j + ny * k)
                s2 = slice(e2 * q2, (e2 + 1) * q2)
                s3 = slice(e3 * q3, (e3 + 1) * q3)
                key = {(round(a, 9), round(b, 9)): t for t, (a, b) in enumerate(zip(x2[s2], y2[s2]))}
                idx = np.array([key[(round(a, 9), round(b, 9))] for a, b in zip(x3[s3], y3[s3])])
                for f3, f2 in ((0, 0), (1, 1), (2, 2), (4, 3)):
                    d = np.abs(U3[f3][s3] - U2[f2][s2][idx]).max() / max(1.0, np.abs(U2[f2]).max())
                    worst = max(worst, d)
                worst = max(worst, np.abs(U3[3][s3]).max())
    return worst


@pytest.mark.parametrize("inttype,steps", [(4, 3), (14, 2)])
def test_roe3d_reduces_to_roe2d(inttype, steps):
    nx, ny, p = 4, 3, 3
    m2 = dgm_io.box_mesh(2, (nx, ny), -5.0, 5.0, p)
    m3 = dgm_io.box_mesh(3, (nx, ny, 2), (-5.0, -5.0, 0.0), (5.0, 5.0, 1.0), p)
    P2 = oracle.Problem(m2, oracle.EULER2D, flux="roe")
    P3 = oracle.Problem(m3, oracle.EULER3D, flux="roe")
    x2, y2, _ = P2.coords()
    x3, y3, z3 = P3.coords()
    f2 = ics.isentropic_vortex(x2, y2, beta=5.0, period=(10.0, 10.0))
    g = ics.isentropic_vortex(x3, y3, beta=5.0, period=(10.0, 10.0))
    f3 = np.stack([g[0], g[1], g[2], np.zeros_like(g[0]), g[3]])
    P2.set_state(P2.project(f2))
    P3.set_state(P3.project(f3))
    assert P2.advance(inttype, 0.01, steps) == 0 and P3.advance(inttype, 0.01, steps) == 0
    assert _by_element_xy(P2, m2, P3, m3, P2.state(), P3.state(), nx, ny) < 1e-12
    # and Roe differs from Lax-Friedrichs on this case (the comparison has teeth)
    L3 = oracle.Problem(m3, oracle.EULER3D, flux="laxfriedrichs")
    L3.set_state(L3.project(f3))
    L3.advance(inttype, 0.01, steps)
    assert np.abs(L3.state() - P3.state()).max() > 1e-6


def test_roe3d_turns_with_the_box():
    """The same Taylor-Green flow on a box and on the box with x, y, z
    relabelled (z, x, y): the Roe run gives the relabelled state."""
    n, p = (3, 2, 2), 2
    m = dgm_io.box_mesh(3, n, 0.0, 2 * np.pi, p)
    nr = (n[2], n[0], n[1])
    mr = dgm_io.box_mesh(3, nr, 0.0, 2 * np.pi, p)
    P = oracle.Problem(m, oracle.EULER3D, flux="roe")
    R = oracle.Problem(mr, oracle.EULER3D, flux="roe")
    x, y, z = P.coords()
    xr, yr, zr = R.coords()
    f = ics.taylor_green(x, y, z, Ma=0.3)
    # the flow in the relabelled frame: new (x, y, z) = old (z, x, y)
    fo = ics.taylor_green(yr, zr, xr, Ma=0.3)
    fr = np.stack([fo[0], fo[3], fo[1], fo[2], fo[4]])
    P.set_state(P.project(f))
    R.set_state(R.project(fr))
    P.advance(4, 0.01, 2)
    R.advance(4, 0.01, 2)
    S, T = P.state(), R.state()
    # element (i, j, k) is element (k, i, j) of the relabelled box; inside
    # an element, points pair up through (x, y, z) <-> (y', z', x')
    q = len(x) // m.ne
    worst = 0.0
    for k in range(n[2]):
        for j in range(n[1]):
            for i in range(n[0]):
                e = i + n[0] * (j + n[1] * k)
                er = k + nr[0] * (i + nr[1] * j)
                key = {(round(yr[t], 9), round(zr[t], 9), round(xr[t], 9)): t for t in range(er * q, (er + 1) * q)}
                for t in range(e * q, (e + 1) * q):
                    u = key[(round(x[t], 9), round(y[t], 9), round(z[t], 9))]
                    worst = max(worst, abs(S[0][t] - T[0][u]), abs(S[1][t] - T[2][u]), abs(S[2][t] - T[3][u]),
                                abs(S[3][t] - T[1][u]), abs(S[4][t] - T[4][u]) / 100.0)
    assert worst < 1e-10
