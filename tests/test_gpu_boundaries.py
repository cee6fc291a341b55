"""GPU parity with boundary sides: Euler 2-D/3-D slip walls, Navier-Stokes
2-D/3-D isothermal walls and the channel's bulk-flow hold, through the C ABI,
against the CPU oracle (which is pinned to the reference's runs/chan golden
restart).

Bar: relative L2 <= 1e-12 against the oracle; the channel run also passes
dgm_diff against the golden restart at the case's own tolerances.
"""
import os
import tempfile

import numpy as np
import pytest

import oracle
from oracle import dgm_io, ics
from tests.cases import (BC_ISOTHERMAL_WALL, BC_SLIP_WALL, BC_STATE, BC_SUBSONIC_OUTFLOW,
                         BC_SUPERSONIC_OUTFLOW, diff_norms, load_wall_golden, passes_dgm_diff)

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def wall_records(n, kind, a=0.0, b=0.0):
    """z- faces of the bottom layer and z+ faces of the top layer of an
    n[0] x n[1] x n[2] box (element index i + nx (j + ny k))."""
    nx, ny, nz = n
    rec = []
    for j in range(ny):
        for i in range(nx):
            rec.append((i + nx * j, 0, kind, a, b))
            rec.append((i + nx * (j + ny * (nz - 1)), 5, kind, a, b))
    return rec


def channel_ic(x, y, z):
    """A wall-bounded perturbed shear flow on [0,2pi]^2 x [0,2] (rho ~ 1,
    Mach ~ 0.1)."""
    u = 1.5 * z * (2.0 - z) + 0.2 * np.sin(x) * np.cos(y) * np.sin(np.pi * z / 2.0)
    v = 0.1 * np.cos(x) * np.sin(2.0 * y)
    w = 0.1 * np.sin(x + y) * np.sin(np.pi * z / 2.0)
    r = 1.0 + 0.01 * np.cos(x) * np.cos(z)
    p = 71.43 + 0.05 * np.sin(y)
    return np.stack([r, r * u, r * v, r * w, p / 0.4 + 0.5 * r * (u * u + v * v + w * w)])


CASES = [
    # name, physics, n, p, flux, inttype, dt, steps, vis, kind, (a, b), hold
    ("euler3d-slip-lf-lsrk14", 8, (3, 2, 3), 3, "laxfriedrichs", 14, 0.002, 2, 0.0, BC_SLIP_WALL, (0, 0), False),
    ("euler3d-slip-roe-rk4", 8, (2, 3, 3), 3, "roe", 4, 0.002, 2, 0.0, BC_SLIP_WALL, (0, 0), False),
    ("euler3d-slip-lf-tvd3-p4", 8, (2, 2, 3), 4, "laxfriedrichs", 3, 0.001, 3, 0.0, BC_SLIP_WALL, (0, 0), False),
    ("ns3d-isothermal-tvd3", 9, (2, 2, 3), 3, "laxfriedrichs", 3, 0.001, 3, 0.02, BC_ISOTHERMAL_WALL,
     (1.0, 178.575), False),
    ("ns3d-isothermal-hold-lsrk14", 9, (3, 2, 3), 3, "laxfriedrichs", 14, 0.001, 2, 0.02, BC_ISOTHERMAL_WALL,
     (1.0, 178.575), True),
    ("ns3d-isothermal-hold-rk4-p2", 9, (2, 3, 4), 2, "laxfriedrichs", 4, 0.001, 2, 0.01, BC_ISOTHERMAL_WALL,
     (1.05, 178.575), True),
    # p = 7, q = 9: the FP64 gradient kernel's two-CTA tile, which reads the
    # wall sides' ghost traces from global memory
    ("ns3d-isothermal-tvd3-p7", 9, (2, 2, 2), 7, "laxfriedrichs", 3, 0.0002, 1, 0.02, BC_ISOTHERMAL_WALL,
     (1.0, 178.575), False),
]


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_walls_match_oracle(case):
    import dgm_b200
    _, phys, n, p, flux, inttype, dt, steps, vis, kind, (a, b), hold = case
    m = dgm_b200.meshgen.box(3, n, (0.0, 0.0, 0.0), (2 * np.pi, 2 * np.pi, 2.0), p)
    rec = wall_records(n, kind, a, b)
    P = oracle.Problem(dgm_io.Mesh(3, m.verts, m.con, m.porder, m.qorder), phys, flux=flux, vis=vis)
    P.set_bc(rec)
    P.set_hold_bulk(hold)
    D = dgm_b200.Domain(m, phys, flux=flux, inttype=inttype, vis=vis, boundaries=rec, bulk_hold=hold)
    x, y, z = P.coords()
    f = channel_ic(x, y, z)
    U0 = P.project(f)
    F_o, F_g = P.rhs(U0), D.time_derivative(U0)
    scale = np.sqrt((F_o ** 2).sum()) + np.sqrt((U0 ** 2).sum())
    assert np.sqrt(((F_g - F_o) ** 2).sum()) / scale < 1e-12
    P.set_state(U0)
    D.set_state(f)
    assert P.advance(inttype, dt, steps) == 0
    D.advance(dt, steps)
    assert rel(D.state(), P.state()) < 1e-12
    # the walls matter: the periodic run of the same case differs
    Q = oracle.Problem(dgm_io.Mesh(3, m.verts, m.con, m.porder, m.qorder), phys, flux=flux, vis=vis)
    Q.set_state(U0)
    Q.advance(inttype, dt, steps)
    assert rel(Q.state(), P.state()) > 1e-9


def wall_records_2d(n, kind, a=0.0, b=0.0):
    """y- sides of the bottom row and y+ sides of the top row of an
    n[0] x n[1] Quad box (element index i + nx j; Quad sides 0 y-, 2 y+)."""
    nx, ny = n
    rec = []
    for i in range(nx):
        rec.append((i, 0, kind, a, b))
        rec.append((i + nx * (ny - 1), 2, kind, a, b))
    return rec


def channel_ic_2d(x, y):
    """A wall-bounded perturbed shear flow on [0,2pi] x [0,2] (Mach ~ 0.1)."""
    u = 1.5 * y * (2.0 - y) + 0.2 * np.sin(x) * np.sin(np.pi * y / 2.0)
    v = 0.1 * np.cos(x) * np.sin(np.pi * y / 2.0)
    r = 1.0 + 0.01 * np.cos(x) * np.cos(y)
    p = 71.43 + 0.05 * np.sin(x)
    return np.stack([r, r * u, r * v, p / 0.4 + 0.5 * r * (u * u + v * v)])


CASES_2D = [
    # name, physics, n, p, flux, inttype, dt, steps, vis, kind, (a, b)
    ("euler2d-slip-lf-lsrk14", 1, (4, 3), 4, "laxfriedrichs", 14, 0.002, 2, 0.0, BC_SLIP_WALL, (0, 0)),
    ("euler2d-slip-roe-tvd3", 1, (3, 4), 3, "roe", 3, 0.002, 3, 0.0, BC_SLIP_WALL, (0, 0)),
    ("ns2d-isothermal-rk4", 2, (4, 3), 3, "laxfriedrichs", 4, 0.001, 3, 0.02, BC_ISOTHERMAL_WALL, (1.0, 178.575)),
    ("ns2d-isothermal-lsrk14-p5", 2, (3, 3), 5, "laxfriedrichs", 14, 0.0005, 2, 0.01, BC_ISOTHERMAL_WALL,
     (1.1, 178.575)),
]


def test_shallow_water_walls_match_oracle():
    """A Gaussian bump of water between two walls (y = -2, 2), periodic in
    x; the balance quirk off (with it on, a still bump would not move)."""
    import dgm_b200
    n, p = (4, 4), 3
    m = dgm_b200.meshgen.box(2, n, (-2.0, -2.0), (2.0, 2.0), p)
    rec = wall_records_2d(n, BC_SLIP_WALL)
    P = oracle.Problem(dgm_io.Mesh(2, m.verts, m.con, m.porder, m.qorder), oracle.SHALLOW)
    P.set_sw_balance(False)
    P.set_bc(rec)
    D = dgm_b200.Domain(m, dgm_b200.SHALLOW, inttype=14, sw_balance=False, boundaries=rec)
    x, y, _ = P.coords()
    f = ics.gaussian_bump(x, y - 1.0, a=0.3, w=0.5)
    U0 = P.project(f)
    F_o, F_g = P.rhs(U0), D.time_derivative(U0)
    scale = np.sqrt((F_o ** 2).sum()) + np.sqrt((U0 ** 2).sum())
    assert np.sqrt(((F_g - F_o) ** 2).sum()) / scale < 1e-12
    P.set_state(U0)
    D.set_state(f)
    assert P.advance(14, 0.001, 5) == 0
    D.advance(0.001, 5)
    assert rel(D.state(), P.state()) < 1e-12


@pytest.mark.parametrize("case", CASES_2D, ids=[c[0] for c in CASES_2D])
def test_walls_2d_match_oracle(case):
    import dgm_b200
    _, phys, n, p, flux, inttype, dt, steps, vis, kind, (a, b) = case
    m = dgm_b200.meshgen.box(2, n, (0.0, 0.0), (2 * np.pi, 2.0), p)
    rec = wall_records_2d(n, kind, a, b)
    P = oracle.Problem(dgm_io.Mesh(2, m.verts, m.con, m.porder, m.qorder), phys, flux=flux, vis=vis)
    P.set_bc(rec)
    D = dgm_b200.Domain(m, phys, flux=flux, inttype=inttype, vis=vis, boundaries=rec)
    x, y, _ = P.coords()
    f = channel_ic_2d(x, y)
    U0 = P.project(f)
    F_o, F_g = P.rhs(U0), D.time_derivative(U0)
    scale = np.sqrt((F_o ** 2).sum()) + np.sqrt((U0 ** 2).sum())
    assert np.sqrt(((F_g - F_o) ** 2).sum()) / scale < 1e-12
    P.set_state(U0)
    D.set_state(f)
    assert P.advance(inttype, dt, steps) == 0
    D.advance(dt, steps)
    assert rel(D.state(), P.state()) < 1e-12
    Q = oracle.Problem(dgm_io.Mesh(2, m.verts, m.con, m.porder, m.qorder), phys, flux=flux, vis=vis)
    Q.set_state(U0)
    Q.advance(inttype, dt, steps)
    assert rel(Q.state(), P.state()) > 1e-9


def _state(nf, u):
    """A uniform state of density 1, x-velocity u and pressure 71.43."""
    v = [1.0, u] + [0.0] * (nf - 3) + [71.43 / 0.4 + 0.5 * u * u]
    return tuple(v)


INOUT = [
    # name, physics, dim, n, p, flux, inttype, dt, steps, vis, walls, outflow kind
    ("euler3d-state-in-out-slip", 8, 3, (3, 2, 3), 3, "laxfriedrichs", 14, 0.002, 2, 0.0, BC_SLIP_WALL, BC_STATE),
    ("ns3d-state-in-out-isothermal", 9, 3, (3, 2, 2), 3, "laxfriedrichs", 3, 0.001, 3, 0.02, BC_ISOTHERMAL_WALL,
     BC_STATE),
    ("euler2d-state-subsonic-out", 1, 2, (4, 3), 4, "roe", 4, 0.002, 3, 0.0, BC_SLIP_WALL, BC_SUBSONIC_OUTFLOW),
    ("euler2d-state-supersonic-out", 1, 2, (4, 3), 3, "laxfriedrichs", 14, 0.002, 2, 0.0, BC_SLIP_WALL,
     BC_SUPERSONIC_OUTFLOW),
    ("ns2d-state-subsonic-out", 2, 2, (4, 3), 3, "laxfriedrichs", 3, 0.001, 3, 0.02, BC_ISOTHERMAL_WALL,
     BC_SUBSONIC_OUTFLOW),
]


@pytest.mark.parametrize("case", INOUT, ids=[c[0] for c in INOUT])
def test_inflow_outflow_match_oracle(case):
    """A fixed-state inflow at x-, an outflow (or a second fixed state in
    3-D) at x+ and walls on the other pair: GPU against the oracle."""
    import dgm_b200
    _, phys, dim, n, p, flux, inttype, dt, steps, vis, wall, out = case
    nf = 5 if dim == 3 else 4
    hi = (2 * np.pi, 2 * np.pi, 2.0) if dim == 3 else (2 * np.pi, 2.0)
    m = dgm_b200.meshgen.box(dim, n, (0.0,) * dim, hi, p)
    wpar = (1.0, 178.575) if wall == BC_ISOTHERMAL_WALL else ()
    if dim == 3:
        rec = [r[:3] + wpar for r in wall_records(n, wall)]
        nx, ny, nz = n
        xm = [i + nx * (j + ny * k) for k in range(nz) for j in range(ny) for i in [0]]
        xp = [i + nx * (j + ny * k) for k in range(nz) for j in range(ny) for i in [nx - 1]]
        rec += [(e, 4, BC_STATE) + _state(nf, 1.0) for e in xm]
        rec += [(e, 2, BC_STATE) + _state(nf, 0.9) for e in xp]
        P = oracle.Problem(dgm_io.Mesh(3, m.verts, m.con, m.porder, m.qorder), phys, flux=flux, vis=vis)
        x, y, z = P.coords()
        f = channel_ic(x, y, z)
    else:
        rec = [r[:3] + wpar for r in wall_records_2d(n, wall)]
        nx, ny = n
        rec += [(i + nx * j, 3, BC_STATE) + _state(nf, 1.0) for j in range(ny) for i in [0]]
        opar = (0.1,) if out == BC_SUBSONIC_OUTFLOW else ()
        rec += [(i + nx * j, 1, out) + opar for j in range(ny) for i in [nx - 1]]
        P = oracle.Problem(dgm_io.Mesh(2, m.verts, m.con, m.porder, m.qorder), phys, flux=flux, vis=vis)
        x, y, _ = P.coords()
        f = channel_ic_2d(x, y)
    P.set_bc(rec)
    D = dgm_b200.Domain(m, phys, flux=flux, inttype=inttype, vis=vis, boundaries=rec)
    U0 = P.project(f)
    F_o, F_g = P.rhs(U0), D.time_derivative(U0)
    scale = np.sqrt((F_o ** 2).sum()) + np.sqrt((U0 ** 2).sum())
    assert np.sqrt(((F_g - F_o) ** 2).sum()) / scale < 1e-12
    P.set_state(U0)
    D.set_state(f)
    assert P.advance(inttype, dt, steps) == 0
    D.advance(dt, steps)
    assert rel(D.state(), P.state()) < 1e-12


def test_channel_golden_on_gpu():
    """runs/chan through the GPU: 512 hexes at p=3, isothermal walls,
    bulk-flow hold, 100 TVD-RK3 steps from the restart initial condition;
    dgm_diff against chan.ref at aeps 5e-10 / reps 1e-8, and 1e-12 against
    the oracle's run."""
    import dgm_b200
    mesh, meta, modal, ic_modal, rec = load_wall_golden("chan")
    inp = meta["inp"]
    D = dgm_b200.Domain(mesh, dgm_b200.NS3D, inttype=inp["inttype"], vis=float(inp["vis"]),
                        boundaries=rec, bulk_hold=True)
    D.set_modes(ic_modal)
    D.advance(float(inp["dt"]), int(inp["Nt"]))
    P = oracle.Problem(mesh, inp["eqntype"], vis=float(inp["vis"]))
    G = D.state()
    norms = diff_norms(G, P.backward(modal), P.wj())
    assert passes_dgm_diff(norms, meta["aeps"], meta["reps"]), norms
    P.set_bc(rec)
    P.set_hold_bulk(True)
    P.set_state(P.backward(ic_modal))
    P.advance(inp["inttype"], float(inp["dt"]), int(inp["Nt"]))
    assert rel(G, P.state()) < 1e-12


def _write_case(root, mesh, meta, tags, sides):
    """The channel case as DGM input files (.inp/.msh/.con/.bc/.bct/.chn)."""
    inp = meta["inp"]
    with open(root + ".inp", "w") as f:
        for k in ("eqntype", "inttype", "dt", "Nt", "p", "vis"):
            f.write(f"{k} = {inp[k]}\n")
    with open(root + ".msh", "w") as f:
        f.write("**MESH DATA**\n%d 3 NE NSD\n" % mesh.ne)
        for e in range(mesh.ne):
            f.write("ELEMENT %d  HEX\n" % e)
            for c in range(3):
                f.write(" ".join("%.17g" % v for v in mesh.verts[e, :, c]) + "\n")
    with open(root + ".con", "w") as f:
        f.write("**CONNECTIVITY DATA**\n%d ne\n" % mesh.ne)
        for r in mesh.con:
            f.write("E %d %d %d %d\n" % tuple(int(v) for v in r))
    with open(root + ".bc", "w") as f:
        f.write("# BOUNDARY CONDITION DATA\n%d nbc\n" % len(tags))
        for t, (e, s) in zip(tags, sides):
            f.write("%s %d %d\n" % (t, e, s))
    with open(root + ".bct", "w") as f:
        for tag, (code, vals) in meta["bct"].items():
            f.write("%s %s\n{\n  %s\n}\n\n" % (code, tag, " ".join("%.17g" % v for v in vals)))
    with open(root + ".chn", "w") as f:
        f.write('{\n  "Nx" : 8,\n  "Ny" : 8,\n  "Nz" : 8\n}\n')


def test_channel_from_files_equals_explicit_boundaries():
    """dgmx_create_from_files reads .bc/.bct/.chn as the reference does: the
    file-built channel steps exactly like the one built from records."""
    import dgm_b200
    mesh, meta, modal, ic_modal, rec = load_wall_golden("chan")
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "chan.npz"))
    inp = meta["inp"]
    with tempfile.TemporaryDirectory() as d:
        root = os.path.join(d, "chan")
        _write_case(root, mesh, meta, meta["bc_tags"], z["bc_sides"])
        F = dgm_b200.Domain.from_files(root, inttype=dgm_b200.TVD3, physics=dgm_b200.NS3D)
    D = dgm_b200.Domain(mesh, dgm_b200.NS3D, inttype=inp["inttype"], vis=float(inp["vis"]),
                        boundaries=rec, bulk_hold=True)
    for X in (F, D):
        X.set_modes(ic_modal)
        X.advance(float(inp["dt"]), 5)
    assert np.array_equal(F.modes(), D.modes())


def test_boundary_domains_refuse_what_is_not_built():
    import dgm_b200
    m = dgm_b200.meshgen.box(3, (2, 2, 2), 0.0, 2 * np.pi, 3)
    rec = wall_records((2, 2, 2), BC_ISOTHERMAL_WALL, 1.0, 100.0)
    with pytest.raises(dgm_b200.DgmxError):   # isothermal wall on Euler
        dgm_b200.Domain(m, dgm_b200.EULER3D, boundaries=rec)
    with pytest.raises(dgm_b200.DgmxError):   # boundaries in the mixed form
        dgm_b200.Domain(m, dgm_b200.EULER3D, precision=dgm_b200.MIXED,
                        boundaries=wall_records((2, 2, 2), BC_SLIP_WALL))
    with pytest.raises(dgm_b200.DgmxError):   # a wall whose partner side stays interior
        dgm_b200.Domain(m, dgm_b200.EULER3D, boundaries=[(0, 0, BC_SLIP_WALL, 0, 0)])
    D = dgm_b200.Domain(m, dgm_b200.EULER3D, boundaries=wall_records((2, 2, 2), BC_SLIP_WALL))
    n = D.variant_count()
    kinds = []
    for i in range(n):
        try:
            kinds.append(D.set_variant(i)[1])
        except dgm_b200.DgmxError:
            kinds.append(2)
    rows, pick = D.autotune(reps=2)
    assert kinds[pick] == 0
