"""GPU parity at the benchmark configurations' own sizes.

The plain FP64 path against the FP64 oracle, per conserved field, on the
meshes, orders, fluxes and integrators the benchmark quotes:

  * the 2-D isentropic vortex: periodic [-5,5]^2, 16 x 16 Quads, p=4 with the
    reference's default q=p+2, beta=5, Lax-Friedrichs, dt from CFL 0.5,
    200 steps of LSRK14 and of the classic RK4 (inttype 4);
  * the 3-D Euler Taylor-Green vortex: periodic [0,2pi]^3, 32^3 Hex, p=3
    (q=5), Mach 0.1, LSRK14, 10 steps, with the Lax-Friedrichs flux (the
    reference's Euler3d flux, src/Euler3d.cpp:584-817, pinned by the golden
    runs/vhex.ref through the oracle) and with the Roe flux (the benchmark's);
  * the 3-D Navier-Stokes Taylor-Green vortex: 24^3 Hex, p=7, q=9, Re=1600,
    Pr=0.71, Mach 0.1, Roe, LSRK14, one step.

Bar: relative L2 <= 1e-12 per conserved field.  The z-momentum of the
Taylor-Green vortex starts at exactly zero and after a few steps is ~2e-3 of
the other momenta, so a relative figure of that field alone measures
round-off against a near-zero norm; it is checked against the norm of the
momentum vector (the three momenta as one field), and its own relative figure
is printed.  The oracle uses every host core.
"""
import math
import os

import numpy as np
import pytest

import oracle
from oracle import dgm_io, ics

pytestmark = pytest.mark.gpu

TOL = 1e-12


def rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def per_field(G, O):
    return [rel(G[k], O[k]) for k in range(G.shape[0])]


def momentum_rel(G, O, dim):
    m = slice(1, 1 + dim)
    return rel(G[m], O[m])


def cfl_dt(U, h, p, dim, gamma=1.4, cfl=0.5):
    r = U[0]
    vel2 = sum((U[1 + i] / r) ** 2 for i in range(dim))
    pr = (gamma - 1.0) * (U[dim + 1] - 0.5 * r * vel2)
    smax = float(np.max(np.sqrt(vel2) + np.sqrt(gamma * pr / r)))
    return cfl * h / ((2 * p + 1) * smax)


@pytest.fixture(scope="module", autouse=True)
def _threads():
    oracle.set_threads(os.cpu_count() or 1)


@pytest.mark.parametrize("inttype", [14, 4], ids=["lsrk14", "rk4"])
def test_vortex2d_16x16_p4_200_steps(inttype):
    import dgm_b200
    n, p, steps = 16, 4, 200
    m = dgm_b200.meshgen.box(2, (n, n), -5.0, 5.0, p)
    assert int(m.qorder[0]) == p + 2
    P = oracle.Problem(dgm_io.Mesh(2, m.verts, m.con, m.porder, m.qorder), oracle.EULER2D, flux="laxfriedrichs")
    D = dgm_b200.Domain(m, dgm_b200.EULER2D, flux="laxfriedrichs", inttype=inttype)
    x, y, _ = P.coords()
    f = ics.isentropic_vortex(x, y, beta=5.0, period=(10.0, 10.0))
    dt = cfl_dt(f, 10.0 / n, p, 2)
    P.set_state(P.project(f))
    D.set_state(f)
    assert P.advance(inttype, dt, steps) == 0
    D.advance(dt, steps)
    G, O = D.state(), P.state()
    errs = per_field(G, O)
    print(f"vortex2d inttype {inttype}: dt {dt:.4e}, per-field rel L2 {['%.2e' % e for e in errs]}")
    assert max(errs) < TOL, errs
    D.close()


def _tgv32(flux, steps):
    import dgm_b200
    n, p = 32, 3
    m = dgm_b200.meshgen.box(3, (n, n, n), 0.0, 2 * math.pi, p)
    assert int(m.qorder[0]) == 5
    P = oracle.Problem(dgm_io.Mesh(3, m.verts, m.con, m.porder, m.qorder), oracle.EULER3D, flux=flux)
    D = dgm_b200.Domain(m, dgm_b200.EULER3D, flux=flux, inttype=dgm_b200.LSRK14)
    x, y, z = P.coords()
    f = ics.taylor_green(x, y, z, Ma=0.1)
    dt = cfl_dt(f, 2 * math.pi / n, p, 3)
    D.set_state(f)
    D.autotune(reps=3)     # the tile the benchmark would run
    P.set_state(P.project(f))
    D.set_state(f)
    assert P.advance(14, dt, steps) == 0
    D.advance(dt, steps)
    G, O = D.state(), P.state()
    D.close()
    return G, O


@pytest.mark.parametrize("flux", ["laxfriedrichs", "roe"])
def test_taylor_green_32cubed_p3_10_steps(flux):
    G, O = _tgv32(flux, 10)
    errs, em = per_field(G, O), momentum_rel(G, O, 3)
    print(f"tgv32 {flux}: per-field rel L2 {['%.2e' % e for e in errs]}, momentum vector {em:.2e}, "
          f"|rho w| / |momentum| {np.linalg.norm(O[3]) / np.linalg.norm(O[1:4]):.2e}")
    for k in (0, 1, 2, 4):
        assert errs[k] < TOL, (k, errs)
    assert em < TOL
    # z-momentum against the momentum vector's norm
    assert np.linalg.norm(G[3] - O[3]) / np.linalg.norm(O[1:4]) < TOL


def test_navier_stokes_taylor_green_24cubed_p7_q9_one_step():
    import dgm_b200
    n, p, q = 24, 7, 9
    m = dgm_b200.meshgen.box(3, (n, n, n), 0.0, 2 * math.pi, p, q)
    P = oracle.Problem(dgm_io.Mesh(3, m.verts, m.con, m.porder, m.qorder), oracle.NS3D, flux="roe",
                       vis=1.0 / 1600.0, Pr=0.71)
    D = dgm_b200.Domain(m, dgm_b200.NS3D, flux="roe", inttype=dgm_b200.LSRK14, vis=1.0 / 1600.0, Pr=0.71)
    x, y, z = P.coords()
    f = ics.taylor_green(x, y, z, Ma=0.1)
    dt = cfl_dt(f, 2 * math.pi / n, p, 3)
    P.set_state(P.project(f))
    D.set_state(f)
    assert P.advance(14, dt, 1) == 0
    D.advance(dt, 1)
    G, O = D.state(), P.state()
    errs, em = per_field(G, O), momentum_rel(G, O, 3)
    print(f"ns tgv24 p7: per-field rel L2 {['%.2e' % e for e in errs]}, momentum vector {em:.2e}")
    for k in (0, 1, 2, 4):
        assert errs[k] < TOL, (k, errs)
    assert em < TOL
    assert np.linalg.norm(G[3] - O[3]) / np.linalg.norm(O[1:4]) < TOL
    D.close()
