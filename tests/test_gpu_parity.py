"""GPU parity: the sm_100a kernels (through the C ABI) against the CPU oracle.

Every case builds the same periodic box mesh for both, evaluates
Domain::time_derivative on the same projected initial condition and advances
the same number of steps.  Bar: relative L2 <= 1e-12 for the advanced state
(FP64 end to end); the RHS alone is compared against the size of the state
it is built from, since it is a small difference of large terms (low-Mach
Taylor-Green: p ~ 71, dp ~ 0.06, and div(rho u) vanishes exactly).
"""
import numpy as np
import pytest

import oracle
from oracle import dgm_io, ics

pytestmark = pytest.mark.gpu

TOL_STATE = 1e-12


def rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def build(phys, dim, n, lo, hi, p, q, flux, inttype, sw_balance=True, rotated=False, vis=0.0):
    import dgm_b200
    from tests.cases import rotated_box
    m = rotated_box(dim, n, lo, hi, p, q, seed=3) if rotated else dgm_b200.meshgen.box(dim, n, lo, hi, p, q)
    P = oracle.Problem(dgm_io.Mesh(m.dim, m.verts, m.con, m.porder, m.qorder), phys, flux=flux, vis=vis)
    if phys == oracle.SHALLOW:
        P.set_sw_balance(sw_balance)
    D = dgm_b200.Domain(m, phys, flux=flux, inttype=inttype, sw_balance=sw_balance, vis=vis)
    return P, D


IV = lambda x, y, z: ics.isentropic_vortex(x, y, beta=5.0, period=(10.0, 10.0))
TG = lambda x, y, z: ics.taylor_green(x, y, z, Ma=0.1)
GB = lambda x, y, z: ics.gaussian_bump(x, y, a=0.3, w=0.5)

CASES = [
    # physics, dim, n, lo, hi, p, q, flux, inttype, ic, dt, steps
    ("euler2d-lf-lsrk", 1, 2, (4, 4), -5, 5, 3, 0, "laxfriedrichs", 14, IV, 0.01, 5),
    ("euler2d-lf-tvd", 1, 2, (4, 4), -5, 5, 3, 0, "laxfriedrichs", 3, IV, 0.01, 5),
    ("euler2d-lf-rk4", 1, 2, (4, 4), -5, 5, 3, 0, "laxfriedrichs", 4, IV, 0.01, 5),
    ("euler2d-roe-q=p+1", 1, 2, (4, 4), -5, 5, 4, 5, "roe", 14, IV, 0.01, 5),
    ("euler2d-ragged-p2", 1, 2, (5, 3), -5, 5, 2, 0, "laxfriedrichs", 3, IV, 0.01, 4),
    ("euler2d-p7", 1, 2, (3, 3), -5, 5, 7, 0, "roe", 4, IV, 0.005, 3),
    ("euler3d-lf-lsrk", 8, 3, (3, 3, 3), 0, 2 * np.pi, 3, 0, "laxfriedrichs", 14, TG, 0.002, 3),
    ("euler3d-lf-tvd", 8, 3, (3, 3, 3), 0, 2 * np.pi, 3, 0, "laxfriedrichs", 3, TG, 0.002, 3),
    ("euler3d-roe-ragged", 8, 3, (3, 2, 4), 0, 2 * np.pi, 2, 0, "roe", 14, TG, 0.002, 3),
    ("euler3d-p5-rk4", 8, 3, (2, 2, 2), 0, 2 * np.pi, 5, 0, "laxfriedrichs", 4, TG, 0.001, 2),
    ("euler3d-p7", 8, 3, (2, 2, 2), 0, 2 * np.pi, 7, 0, "laxfriedrichs", 14, TG, 0.0005, 1),
    ("shallow-lsrk", 30, 2, (4, 4), -2, 2, 3, 0, "laxfriedrichs", 14, GB, 0.001, 5),
    ("euler2d-rotated-roe", 1, 2, (4, 3), -5, 5, 3, 0, "roe", 14, IV, 0.01, 4, True),
    ("euler3d-rotated-lf", 8, 3, (3, 3, 3), 0, 2 * np.pi, 3, 0, "laxfriedrichs", 3, TG, 0.002, 3, True),
    ("euler3d-rotated-roe-p4", 8, 3, (2, 3, 2), 0, 2 * np.pi, 4, 0, "roe", 14, TG, 0.001, 2, True),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_rhs_and_advance_match_oracle(case):
    _, phys, dim, n, lo, hi, p, q, flux, inttype, ic, dt, steps = case[:13]
    rotated = len(case) > 13 and case[13]
    sw = phys != oracle.SHALLOW  # exercise shallow water with the balance off here
    P, D = build(phys, dim, n, lo, hi, p, q, flux, inttype, sw_balance=sw, rotated=rotated)
    x, y, z = P.coords()
    xd, yd, zd = D.coordinates()
    assert np.abs(x - xd).max() < 1e-13 and np.abs(y - yd).max() < 1e-13
    f = ic(x, y, z)
    U0 = P.project(f)
    # Domain::time_derivative on host buffers
    F_o, F_g = P.rhs(U0), D.time_derivative(U0)
    # the RHS of a smooth low-Mach flow is a small difference of large
    # fluxes, so it is checked against the state's scale (time unit 1)
    scale = np.sqrt((F_o ** 2).sum()) + np.sqrt((U0 ** 2).sum())
    assert np.sqrt(((F_g - F_o) ** 2).sum()) / scale < 1e-12
    # set_state projects exactly like set_ic + project
    P.set_state(U0)
    D.set_state(f)
    assert rel(D.state(), U0) < TOL_STATE
    assert P.advance(inttype, dt, steps) == 0
    D.advance(dt, steps)
    assert rel(D.state(), P.state()) < TOL_STATE
    # the kernels really ran: one launch per stage
    stages = {14: 14, 3: 3, 4: 4}[inttype]
    assert D.launch_count() >= stages * steps


NS_CASES = [
    # name, physics, dim, n, lo, hi, p, q, flux, inttype, ic, dt, steps, vis, rotated
    ("ns2d-vquad-like", 2, 2, (3, 3), 0, 4, 4, 0, "laxfriedrichs", 3, "vortex", 0.001, 5, 0.02, False),
    ("ns2d-rk4-q=p+1", 2, 2, (4, 3), 0, 4, 3, 4, "laxfriedrichs", 4, "vortex", 0.001, 4, 0.05, False),
    ("ns2d-rotated-roe", 2, 2, (3, 4), 0, 4, 3, 0, "roe", 14, "vortex", 0.001, 3, 0.02, True),
    ("ns2d-p7", 2, 2, (2, 2), 0, 4, 7, 0, "laxfriedrichs", 14, "vortex", 0.0005, 2, 0.01, False),
    ("ns3d-tgv-p3", 9, 3, (3, 3, 3), 0, 2 * np.pi, 3, 0, "laxfriedrichs", 14, "tgv", 0.002, 3, 0.01, False),
    ("ns3d-tvd-p2-ragged", 9, 3, (3, 2, 4), 0, 2 * np.pi, 2, 0, "laxfriedrichs", 3, "tgv", 0.002, 3, 0.05, False),
    ("ns3d-rotated-p4", 9, 3, (2, 3, 2), 0, 2 * np.pi, 4, 0, "laxfriedrichs", 14, "tgv", 0.001, 2, 0.01, True),
    ("ns3d-p7", 9, 3, (2, 2, 2), 0, 2 * np.pi, 7, 0, "laxfriedrichs", 14, "tgv", 0.0005, 1, 1.0 / 1600, False),
    ("ns3d-p7-q=p+1-roe", 9, 3, (2, 2, 2), 0, 2 * np.pi, 7, 8, "roe", 14, "tgv", 0.0005, 1, 1.0 / 1600, False),
    ("ns3d-p3-q=p+1-ragged", 9, 3, (3, 2, 2), 0, 2 * np.pi, 3, 4, "laxfriedrichs", 4, "tgv", 0.002, 2, 0.02, False),
]


@pytest.mark.parametrize("case", NS_CASES, ids=[c[0] for c in NS_CASES])
def test_navier_stokes_br1_matches_oracle(case):
    _, phys, dim, n, lo, hi, p, q, flux, inttype, ic, dt, steps, vis, rotated = case
    P, D = build(phys, dim, n, lo, hi, p, q, flux, inttype, rotated=rotated, vis=vis)
    x, y, z = P.coords()
    if ic == "vortex":
        f = ics.vortex_ic(x, y, [(2.0, 2.0, 0.3, 1.0, 0.5)], nf=4)
    else:
        f = TG(x, y, z)
    U0 = P.project(f)
    F_o, F_g = P.rhs(U0), D.time_derivative(U0)
    scale = np.sqrt((F_o ** 2).sum()) + np.sqrt((U0 ** 2).sum())
    assert np.sqrt(((F_g - F_o) ** 2).sum()) / scale < 1e-12
    P.set_state(U0)
    D.set_state(f)
    assert P.advance(inttype, dt, steps) == 0
    D.advance(dt, steps)
    assert rel(D.state(), P.state()) < TOL_STATE
    # viscosity matters in these cases: the Euler RHS differs
    E = oracle.Problem(dgm_io.Mesh(dim, P.mesh.verts, P.mesh.con, P.mesh.porder, P.mesh.qorder),
                       oracle.EULER2D if dim == 2 else oracle.EULER3D, flux=flux)
    assert rel(E.rhs(U0), F_o) > 1e-8


NS32_CASES = [
    # name, NS physics, its Euler counterpart, dim, n, lo, hi, p, q, inttype, dt, vis
    ("ns3d-p7-q9-tgv", 9, 8, 3, (4, 4, 4), 0, 2 * np.pi, 7, 9, 14, 0.002, 1.0 / 1600),
    ("ns3d-p3-tgv", 9, 8, 3, (8, 8, 8), 0, 2 * np.pi, 3, 0, 3, 0.004, 0.01),
    ("ns2d-p4-vortex", 2, 1, 2, (6, 6), -5, 5, 4, 0, 4, 0.01, 0.02),
]
# FP32 viscous form: bound on its distance from the FP64 path relative to the
# viscous part itself (the FP64 Navier-Stokes result minus the Euler result)
TOL_VISC32 = 2e-4


def stage_weight_rss(inttype):
    """Root-sum-square of a scheme's effective stage weights: the factor by
    which independent per-stage rounding errors of the right-hand side reach
    the step.  LSRK14's 2N-storage coefficients give weights as large as
    37 and -39 (summing to 1), so about 55; TVD3 and RK4 stay below 1."""
    if inttype != 14:
        return 1.0
    A, B = oracle.lsrk14_coefficients()
    w = [sum(B[k] * np.prod(A[j + 1:k + 1]) for k in range(j, 14)) for j in range(14)]
    return float(np.sqrt(np.sum(np.square(w))))


NS32_RUNS = [(c, False) for c in NS32_CASES] + [(NS32_CASES[0], True)]


@pytest.mark.parametrize("case,tensor", NS32_RUNS,
                         ids=[c[0] + ("-3xtf32" if t else "") for c, t in NS32_RUNS])
def test_navier_stokes_fp32_viscous_form(case, tensor):
    """precision = MIXED for Navier-Stokes runs the BR1 gradient and viscous
    kernels in FP32 (stage kernel, registers and traces FP64).  Measured
    against the viscous contribution alone (momentum vector, energy): the
    right-hand side (nodal path) of the FP32 form stays within TOL_VISC32 of
    the FP64 path, and one step (modal path) within TOL_VISC32 times the
    scheme's stage-weight factor; the FP64 path's own parity with the oracle
    is checked on the same step.  Low-Mach Taylor-Green (E/rho ~ 180 against
    |u|^2/2 ~ 0.5) is the case that needs the mean-shifted internal energy.
    `tensor`: the viscous kernels' contractions as 3xTF32 tensor-core
    products (p >= 5), held to the same bars."""
    import dgm_b200
    _, phys, ephys, dim, n, lo, hi, p, q, inttype, dt, vis = case
    m = dgm_b200.meshgen.box(dim, n, lo, hi, p, q)
    D32 = dgm_b200.Domain(m, phys, flux="roe", inttype=inttype, vis=vis, precision=dgm_b200.MIXED)
    if tensor:
        D32.set_tensor_contractions(True)
    D64 = dgm_b200.Domain(m, phys, flux="roe", inttype=inttype, vis=vis)
    D0 = dgm_b200.Domain(m, ephys, flux="roe", inttype=inttype)
    P = oracle.Problem(dgm_io.Mesh(m.dim, m.verts, m.con, m.porder, m.qorder), phys, flux="roe", vis=vis)
    x, y, z = P.coords()
    f = TG(x, y, z) if dim == 3 else ics.vortex_ic(x, y, [(0.0, 0.0, 1.0, 1.0, 0.5)], nf=4)
    U0 = P.project(f)
    F32, F64, F0 = D32.time_derivative(U0), D64.time_derivative(U0), D0.time_derivative(U0)
    for D in (D32, D64, D0):
        D.set_state(f)
        D.advance(dt, 1)
    S32, S64, S0 = D32.state(), D64.state(), D0.state()
    P.set_state(U0)
    assert P.advance(inttype, dt, 1) == 0
    assert rel(S64, P.state()) < TOL_STATE
    # density has no viscous part; the momentum components are measured as
    # one vector (Taylor-Green's w component has none by symmetry)
    for k in (slice(1, dim + 1), slice(dim + 1, dim + 2)):
        rhs = np.linalg.norm(F32[k] - F64[k]) / np.linalg.norm(F64[k] - F0[k])
        step = np.linalg.norm(S32[k] - S64[k]) / np.linalg.norm(S64[k] - S0[k])
        assert rhs < TOL_VISC32 and step < TOL_VISC32 * stage_weight_rss(inttype), (k, rhs, step)
    assert not np.array_equal(S32, S64)
    for D in (D32, D64, D0):
        D.close()


MIXED_CASES = [
    ("euler3d-tgv", 8, 3, (4, 4, 4), 0, 2 * np.pi, 3, "laxfriedrichs", TG, 0.002, 20),
    ("euler3d-roe-p5", 8, 3, (2, 2, 2), 0, 2 * np.pi, 5, "roe", TG, 0.001, 10),
    ("euler2d-vortex", 1, 2, (6, 6), -5, 5, 4, "laxfriedrichs", IV, 0.01, 20),
    ("shallow", 30, 2, (4, 4), -2, 2, 3, "laxfriedrichs", GB, 0.001, 20),
]


@pytest.mark.parametrize("case", MIXED_CASES, ids=[c[0] for c in MIXED_CASES])
def test_mixed_precision_within_1e6_of_fp64_oracle(case):
    """FP32 states, fluxes and contractions with the FP64 solution register
    (LSRK14): relative L2 error against the FP64 oracle stays <= 1e-6."""
    import dgm_b200
    _, phys, dim, n, lo, hi, p, flux, ic, dt, steps = case
    m = dgm_b200.meshgen.box(dim, n, lo, hi, p)
    P = oracle.Problem(dgm_io.Mesh(m.dim, m.verts, m.con, m.porder, m.qorder), phys, flux=flux)
    if phys == oracle.SHALLOW:
        P.set_sw_balance(False)
    D = dgm_b200.Domain(m, phys, flux=flux, inttype=dgm_b200.LSRK14, precision=dgm_b200.MIXED, sw_balance=False)
    x, y, z = P.coords()
    f = ic(x, y, z)
    U0 = P.project(f)
    P.set_state(U0)
    D.set_state(f)
    P.advance(14, dt, steps)
    D.advance(dt, steps)
    err = rel(D.state(), P.state())
    assert err < 1e-6, err
    assert err > 1e-13  # it really ran in FP32
    # the state actually moved by much more than the error
    assert rel(P.state(), U0) > 10 * err


def test_autotune_keeps_results_and_state():
    """The tile autotuner only changes launch shapes: the state is untouched
    by tuning and every variant gives the oracle's answer."""
    P, D = build(oracle.EULER3D, 3, (3, 3, 3), 0, 2 * np.pi, 3, 0, "roe", 14)
    x, y, z = P.coords()
    f = TG(x, y, z)
    U0 = P.project(f)
    D.set_state(f)
    before = D.state()
    rows, pick = D.autotune(reps=3)
    assert len(rows) >= 2 and 0 <= pick < len(rows)
    assert np.array_equal(D.state(), before)
    P.set_state(U0)
    P.advance(14, 0.002, 2)
    D.advance(0.002, 2)
    assert rel(D.state(), P.state()) < TOL_STATE


VARIANT_CASES = [
    # physics, dim, n, lo, hi, p, flux, inttype, ic, dt, steps, precision
    ("euler3d-roe-p3", 8, 3, (3, 2, 3), 0, 2 * np.pi, 3, "roe", 14, TG, 0.002, 2, 0),
    ("euler3d-lf-p4-tvd", 8, 3, (2, 2, 2), 0, 2 * np.pi, 4, "laxfriedrichs", 3, TG, 0.001, 2, 0),
    ("euler3d-lf-p4-lsrk-ragged", 8, 3, (2, 3, 2), 0, 2 * np.pi, 4, "laxfriedrichs", 14, TG, 0.001, 2, 0),
    ("euler3d-roe-p2-lsrk", 8, 3, (3, 3, 2), 0, 2 * np.pi, 2, "roe", 14, TG, 0.002, 2, 0),
    ("euler3d-lf-p3-lsrk-rotated", 8, 3, (3, 2, 3), 0, 2 * np.pi, 3, "laxfriedrichs", 14, TG, 0.002, 2, 0, True),
    ("euler3d-lf-p3-mixed", 8, 3, (3, 2, 3), 0, 2 * np.pi, 3, "laxfriedrichs", 14, TG, 0.002, 2, 1),
    ("euler3d-lf-p5-lsrk-rotated", 8, 3, (2, 2, 2), 0, 2 * np.pi, 5, "laxfriedrichs", 14, TG, 0.001, 2, 0, True),
    ("euler3d-roe-p3-rotated", 8, 3, (3, 2, 3), 0, 2 * np.pi, 3, "roe", 14, TG, 0.002, 2, 0, True),
    ("euler3d-roe-p3-mixed-rotated", 8, 3, (3, 2, 3), 0, 2 * np.pi, 3, "roe", 14, TG, 0.002, 2, 1, True),
    ("euler3d-lf-p5-mixed", 8, 3, (2, 2, 2), 0, 2 * np.pi, 5, "laxfriedrichs", 14, TG, 0.001, 2, 1),
    ("euler2d-roe-p3-rk4", 1, 2, (4, 3), -5, 5, 3, "roe", 4, IV, 0.01, 3, 0),
    ("shallow-p2", 30, 2, (4, 4), -2, 2, 2, "laxfriedrichs", 14, GB, 0.001, 3, 0),
    ("ns3d-p3", 9, 3, (2, 2, 2), 0, 2 * np.pi, 3, "laxfriedrichs", 14, TG, 0.002, 2, 0),
    ("euler3d-roe-p3-mixed", 8, 3, (3, 2, 3), 0, 2 * np.pi, 3, "roe", 14, TG, 0.002, 2, 1),
    ("euler2d-p5-mixed", 1, 2, (3, 3), -5, 5, 5, "laxfriedrichs", 14, IV, 0.005, 3, 1),
]


@pytest.mark.parametrize("case", VARIANT_CASES, ids=[c[0] for c in VARIANT_CASES])
def test_every_tile_variant_matches_oracle(case):
    """Every compiled tile of the stage kernel -- elements per CTA, register
    caps, and the prefetching persistent kernel where the block sizes allow
    it -- gives the oracle's answer (FP64: 1e-12; mixed form: 1e-6)."""
    import dgm_b200
    _, phys, dim, n, lo, hi, p, flux, inttype, ic, dt, steps, prec = case[:13]
    rotated = len(case) > 13 and case[13]
    from tests.cases import rotated_box
    m = rotated_box(dim, n, lo, hi, p, 0, seed=3) if rotated else dgm_b200.meshgen.box(dim, n, lo, hi, p)
    vis = 0.05 if phys == oracle.NS3D else 0.0
    P = oracle.Problem(dgm_io.Mesh(m.dim, m.verts, m.con, m.porder, m.qorder), phys, flux=flux, vis=vis)
    if phys == oracle.SHALLOW:
        P.set_sw_balance(False)
    x, y, z = P.coords()
    f = ic(x, y, z)
    P.set_state(P.project(f))
    P.advance(inttype, dt, steps)
    ref = P.state()
    D = dgm_b200.Domain(m, phys, flux=flux, inttype=inttype, sw_balance=False, vis=vis, precision=prec)
    count = D.variant_count()
    assert count >= 2
    kinds = set()
    for k in range(count):
        _, kind = D.set_variant(k)
        kinds.add(kind)
        D.set_state(f)
        D.advance(dt, steps)
        err = rel(D.state(), ref)
        assert err < (1e-6 if prec else TOL_STATE), (k, kind, err)
    if phys == oracle.EULER3D and p == 3:
        assert 2 in kinds       # the prefetching kernel is built for this case
    if phys == oracle.EULER3D and 2 <= p <= 5:
        assert 3 in kinds       # the second-form stage kernel is built for this case


def test_shallow_balance_keeps_state_steady():
    """REO_SHALLOW_ENFORCE_BALANCE subtracts the first RHS (src/Shallow.cpp:255-267),
    so the bump stays exactly where it is on both sides."""
    P, D = build(oracle.SHALLOW, 2, (4, 4), -2, 2, 3, 0, "laxfriedrichs", 4, sw_balance=True)
    x, y, z = P.coords()
    U0 = P.project(GB(x, y, z))
    P.set_state(U0)
    D.set_state(U0)
    P.advance(4, 0.001, 4)
    D.advance(0.001, 4)
    assert rel(D.state(), P.state()) < TOL_STATE
    assert rel(D.state(), U0) < 1e-13


def test_conservation():
    """Periodic mesh.  Mass has a linear flux and is conserved to round-off.
    Momentum and energy drift by the aliasing the reference scheme carries
    (the volume term differentiates the GLL interpolant of F(U) while the
    lift subtracts F of the Gauss-point trace, src/Euler3d.cpp:720-724 and
    src/Hex.cpp:1768-1783); that drift must equal the oracle's."""
    import dgm_b200
    m = dgm_b200.meshgen.box(3, (4, 4, 4), 0, 2 * np.pi, 3)
    D = dgm_b200.Domain(m, dgm_b200.EULER3D, inttype=dgm_b200.LSRK14)
    P = oracle.Problem(dgm_io.Mesh(3, m.verts, m.con, m.porder, m.qorder), oracle.EULER3D)
    x, y, z = P.coords()
    f = TG(x, y, z)
    D.set_state(f)
    P.set_state(P.project(f))
    wj = P.wj()
    I0 = D.integrals()
    assert np.allclose(I0, (P.state() * wj).sum(axis=1), rtol=1e-13, atol=1e-12)
    D.advance(0.01, 20)
    P.advance(14, 0.01, 20)
    I1, O1 = D.integrals(), (P.state() * wj).sum(axis=1)
    assert abs(I1[0] - I0[0]) <= 1e-13 * abs(I0[0])
    drift_gpu, drift_oracle = I1 - I0, O1 - I0
    assert np.all(np.abs(drift_gpu - drift_oracle) <= 1e-11 * np.maximum(np.abs(I0), 1.0))


def test_nonphysical_state_is_reported_not_trapped():
    """A negative density on the host makes the C ABI return
    DGMX_ERR_NONPHYSICAL; the handle stays usable afterwards."""
    import dgm_b200
    m = dgm_b200.meshgen.box(2, (3, 3), -5, 5, 2)
    D = dgm_b200.Domain(m, dgm_b200.EULER2D)
    x, y, z = D.coordinates()
    U = IV(x, y, z)
    bad = U.copy()
    bad[0, :] = -1.0
    with pytest.raises(dgm_b200.NonPhysicalState):
        D.time_derivative(bad)
    F = D.time_derivative(U)
    assert np.isfinite(F).all()


def test_unsupported_order_is_an_error():
    import dgm_b200
    m = dgm_b200.meshgen.box(3, (2, 2, 2), 0, 1, 9)
    with pytest.raises(dgm_b200.DgmxError):
        dgm_b200.Domain(m, dgm_b200.EULER3D)
