"""GPU parity of source terms (Source::apply, F -= S before the projection)
for the 2-D physics, against the oracle with the same source field.  The
reference applies sources in Euler::time_derivative (src/Euler.cpp:282-287),
Navier_Stokes::time_derivative (src/Navier_Stokes.cpp:95-100) and
Shallow::time_derivative (src/Shallow.cpp:255-260), where the first
right-hand side kept for the balance includes the source; Euler3d and
Navier_Stokes3d apply none."""
import numpy as np
import pytest

import oracle
from oracle import dgm_io, ics

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def source_field(x, y, nf, scale):
    """A smooth, non-polynomial source: Gaussian bumps per field."""
    return np.stack([scale * (n + 1) * np.exp(-((x - 0.3 * n) ** 2 + (y + 0.2 * n) ** 2)) for n in range(nf)])


CASES = [
    # name, physics, n, lo, hi, p, flux, inttype, vis, sw_balance, ic, dt, steps
    ("euler2d-lf-lsrk14", 1, (6, 6), -5, 5, 4, "laxfriedrichs", 14, 0.0, False, "vortex", 0.01, 10),
    ("euler2d-roe-tvd3", 1, (5, 5), -5, 5, 3, "roe", 3, 0.0, False, "vortex", 0.01, 10),
    ("ns2d-rk4", 2, (5, 5), -5, 5, 4, "laxfriedrichs", 4, 0.02, False, "vortex", 0.005, 10),
    ("shallow-balance-off", 30, (6, 6), -2, 2, 3, "laxfriedrichs", 14, 0.0, False, "bump", 0.001, 10),
    ("shallow-balance-on", 30, (6, 6), -2, 2, 3, "laxfriedrichs", 14, 0.0, True, "bump", 0.001, 10),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_source_parity(case):
    import dgm_b200
    _, phys, n, lo, hi, p, flux, inttype, vis, bal, ic, dt, steps = case
    m = dgm_b200.meshgen.box(2, n, lo, hi, p)
    P = oracle.Problem(dgm_io.Mesh(2, m.verts, m.con, m.porder, m.qorder), phys, flux=flux, vis=vis)
    D = dgm_b200.Domain(m, phys, flux=flux, inttype=inttype, vis=vis, sw_balance=bal)
    if phys == 30:
        P.set_sw_balance(bal)
    x, y, _ = P.coords()
    f = ics.vortex_ic(x, y, [(0.0, 0.0, 1.0, 1.0, 0.5)], nf=4) if ic == "vortex" else \
        ics.gaussian_bump(x, y, a=0.3, w=0.5)
    nf = f.shape[0]
    S = source_field(x, y, nf, 0.05)
    U0 = P.project(f)
    D_plain = dgm_b200.Domain(m, phys, flux=flux, inttype=inttype, vis=vis, sw_balance=bal)
    F_plain = D_plain.time_derivative(U0)
    D_plain.close()
    P.set_source(S)
    D.set_source(S)
    F_g, F_o = D.time_derivative(U0), P.rhs(U0)
    # the right-hand side against the size of the state it is built from
    assert np.linalg.norm(F_g - F_o) <= 1e-12 * np.linalg.norm(U0)
    if not bal:   # with the balance on, a source fixed in time cancels (as in the reference)
        assert not np.allclose(F_g, F_plain)
    P.set_state(U0)
    D.set_state(f)
    assert P.advance(inttype, dt, steps) == 0
    D.advance(dt, steps)
    assert rel(D.state(), P.state()) < 1e-12
    # removing it restores the plain right-hand side
    D.set_source(None)
    D.set_state(f)
    assert np.array_equal(D.time_derivative(U0), F_plain)
    D.close()


def test_source_constant_cancelled_by_balance():
    """ConstSource with the shallow-water balance on: the first right-hand
    side (source included) is kept and subtracted, so a lake at rest stays at
    rest with or without the source, as in the reference."""
    import dgm_b200
    m = dgm_b200.meshgen.box(2, (4, 4), -2, 2, 3)
    D = dgm_b200.Domain(m, dgm_b200.SHALLOW, sw_balance=True)
    x, y, _ = D.coordinates()
    U = np.stack([np.full_like(x, 1.0), 0 * x, 0 * x])
    D.set_source([0.3, 0.1, -0.2])
    D.set_state(U)
    D.advance(0.001, 20)
    assert np.abs(D.state() - U).max() < 1e-13
    D.close()


def test_source_mixed_precision():
    """The mixed form applies the projected source in FP32: within 1e-6 of
    the FP64 oracle, as its other mixed cases."""
    import dgm_b200
    m = dgm_b200.meshgen.box(2, (6, 6), -5, 5, 4)
    P = oracle.Problem(dgm_io.Mesh(2, m.verts, m.con, m.porder, m.qorder), 1)
    D = dgm_b200.Domain(m, dgm_b200.EULER2D, precision=dgm_b200.MIXED)
    x, y, _ = P.coords()
    f = ics.vortex_ic(x, y, [(0.0, 0.0, 1.0, 1.0, 0.5)], nf=4)
    S = source_field(x, y, 4, 0.05)
    P.set_source(S)
    D.set_source(S)
    P.set_state(P.project(f))
    D.set_state(f)
    assert P.advance(14, 0.01, 20) == 0
    D.advance(0.01, 20)
    assert rel(D.state(), P.state()) < 1e-6


def test_source_refused_in_3d():
    import dgm_b200
    m = dgm_b200.meshgen.box(3, (2, 2, 2), 0, 1, 2)
    D = dgm_b200.Domain(m, dgm_b200.EULER3D)
    with pytest.raises(dgm_b200.DgmxError):
        D.set_source(np.zeros((5, D.nq)))
    D.close()


@pytest.mark.parametrize("inttype", [14, 3, 4])
def test_gaussian_source_pulse(inttype):
    """Shallow::GaussianSource: hamp exp(-(x-x0)^2/(2sx^2) - (y-y0)^2/(2sy^2))
    on the height field, times exp(-(t-t0)^2/(2st^2)) at each stage's time,
    against the oracle after 10 steps (the pulse peaks inside the run); the
    domain time then equals 10 dt in both codes."""
    import dgm_b200
    m = dgm_b200.meshgen.box(2, (6, 6), -2, 2, 3)
    P = oracle.Problem(dgm_io.Mesh(2, m.verts, m.con, m.porder, m.qorder), 30)
    D = dgm_b200.Domain(m, dgm_b200.SHALLOW, inttype=inttype, sw_balance=False)
    P.set_sw_balance(False)
    x, y, _ = P.coords()
    f = ics.gaussian_bump(x, y, a=0.3, w=0.5)
    S = np.zeros_like(f)
    S[0] = 0.2 * np.exp(-(x - 0.5) ** 2 / (2 * 0.3 ** 2) - (y + 0.25) ** 2 / (2 * 0.4 ** 2))
    dt = 0.001
    for X in (P, D):
        X.set_source(S)
        X.set_source_pulse(4.5 * dt, 3 * dt)
    P.set_state(P.project(f))
    D.set_state(f)
    assert P.advance(inttype, dt, 10) == 0
    D.advance(dt, 10)
    assert rel(D.state(), P.state()) < 1e-12
    assert abs(D.time() - 10 * dt) < 1e-15 and abs(P.time() - 10 * dt) < 1e-15
    # the factor matters: without it the run differs
    D.set_source_pulse(0.0, 0.0)
    D.set_time(0.0)
    D.set_state(f)
    D.advance(dt, 10)
    assert rel(D.state(), P.state()) > 1e-9
    D.close()
