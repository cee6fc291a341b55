"""Element partitions on the GPU: the in-process group (every part a handle
on one device, the halo exchange by device copies through the same pack /
unpack lists as the NCCL path) steps exactly like the unpartitioned domain,
and like the oracle."""
import numpy as np
import pytest

import oracle
from oracle import dgm_io, ics
from tests.cases import BC_ISOTHERMAL_WALL

pytestmark = pytest.mark.gpu


CASES = [
    # name, physics, dim, n, lo, hi, p, flux, inttype, dt, steps, vis, nparts, kind
    ("euler3d-lsrk14-2-slabs", 8, 3, (3, 2, 4), 0.0, 2 * np.pi, 3, "roe", 14, 0.002, 2, 0.0, 2, "slabs"),
    ("euler3d-tvd3-3-random", 8, 3, (3, 3, 2), 0.0, 2 * np.pi, 2, "laxfriedrichs", 3, 0.002, 3, 0.0, 3, "random"),
    ("ns3d-rk4-4-random", 9, 3, (2, 3, 3), 0.0, 2 * np.pi, 3, "laxfriedrichs", 4, 0.002, 2, 0.02, 4, "random"),
    ("euler2d-lsrk14-3-slabs", 1, 2, (5, 4), -5.0, 5.0, 4, "laxfriedrichs", 14, 0.005, 2, 0.0, 3, "slabs"),
    ("ns2d-tvd3-2-random", 2, 2, (4, 4), 0.0, 4.0, 3, "laxfriedrichs", 3, 0.001, 3, 0.02, 2, "random"),
]


def _ic(phys, x, y, z):
    if phys in (8, 9):
        return ics.taylor_green(x, y, z, Ma=0.1)
    if phys == 2:
        return ics.vortex_ic(x, y, [(2.0, 2.0, 0.3, 1.0, 0.5)], nf=4)
    return ics.isentropic_vortex(x, y, beta=5.0, period=(10.0, 10.0))


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_group_equals_single_domain(case):
    import dgm_b200
    _, phys, dim, n, lo, hi, p, flux, inttype, dt, steps, vis, nparts, kind = case
    m = dgm_b200.meshgen.box(dim, n, lo, hi, p)
    ne = m.verts.shape[0]
    part = ((np.arange(ne) * nparts) // ne if kind == "slabs"
            else np.random.default_rng(5).permutation(np.arange(ne) % nparts))
    D = dgm_b200.Domain(m, phys, flux=flux, inttype=inttype, vis=vis, sw_balance=False)
    G = dgm_b200.Group(m, phys, part, flux=flux, inttype=inttype, vis=vis)
    x, y, z = D.coordinates()
    f = _ic(phys, x, y, z)
    D.set_state(f)
    G.set_state(f)
    assert np.array_equal(G.state(), D.state())
    D.advance(dt, steps)
    G.advance(dt, steps)
    S = D.state()
    assert np.array_equal(G.state(), S)
    P = oracle.Problem(dgm_io.Mesh(m.dim, m.verts, m.con, m.porder, m.qorder), phys, flux=flux, vis=vis)
    P.set_state(P.project(f))
    P.advance(inttype, dt, steps)
    O = P.state()
    assert float(np.sqrt(((S - O) ** 2).sum() / (O ** 2).sum())) < 1e-12
    G.close()


MIXED_CASES = [
    # name, physics, dim, n, lo, hi, p, flux, dt, steps, nparts, kind
    ("euler3d-roe-p3-2-slabs", 8, 3, (4, 4, 4), 0.0, 2 * np.pi, 3, "roe", 0.002, 3, 2, "slabs"),
    ("euler3d-lf-p2-3-random", 8, 3, (3, 3, 2), 0.0, 2 * np.pi, 2, "laxfriedrichs", 0.002, 3, 3, "random"),
    ("euler2d-lf-p4-3-slabs", 1, 2, (5, 4), -5.0, 5.0, 4, "laxfriedrichs", 0.005, 3, 3, "slabs"),
    ("shallow-lf-p3-2-random", 30, 2, (4, 4), -2.0, 2.0, 3, "laxfriedrichs", 0.001, 3, 2, "random"),
]


def _ic_mixed(phys, x, y, z):
    if phys == 30:
        return ics.gaussian_bump(x, y, a=0.3, w=0.5)
    return _ic(phys, x, y, z)


@pytest.mark.parametrize("case", MIXED_CASES, ids=[c[0] for c in MIXED_CASES])
def test_mixed_group_equals_mixed_single_domain(case):
    """The mixed form (FP32 traces, FP64 register, LSRK14) on an element
    partition: every part takes the unpartitioned domain's reference state
    (the integrals summed over the whole mesh in one fixed order), the FP32
    trace blocks cross in the halo, and the state equals the unpartitioned
    mixed domain's bit for bit; it stays within 1e-6 of the FP64 oracle."""
    import dgm_b200
    _, phys, dim, n, lo, hi, p, flux, dt, steps, nparts, kind = case
    m = dgm_b200.meshgen.box(dim, n, lo, hi, p)
    ne = m.verts.shape[0]
    part = ((np.arange(ne) * nparts) // ne if kind == "slabs"
            else np.random.default_rng(7).permutation(np.arange(ne) % nparts))
    D = dgm_b200.Domain(m, phys, flux=flux, inttype=dgm_b200.LSRK14, precision=dgm_b200.MIXED, sw_balance=False)
    G = dgm_b200.Group(m, phys, part, flux=flux, inttype=dgm_b200.LSRK14, precision=dgm_b200.MIXED)
    x, y, z = D.coordinates()
    f = _ic_mixed(phys, x, y, z)
    D.set_state(f)
    G.set_state(f)
    assert np.array_equal(G.state(), D.state())
    D.advance(dt, steps)
    G.advance(dt, steps)
    S = D.state()
    assert np.array_equal(G.state(), S)
    P = oracle.Problem(dgm_io.Mesh(m.dim, m.verts, m.con, m.porder, m.qorder), phys, flux=flux)
    if phys == oracle.SHALLOW:
        P.set_sw_balance(False)
    U0 = P.project(f)
    P.set_state(U0)
    P.advance(14, dt, steps)
    O = P.state()
    err = float(np.sqrt(((S - O) ** 2).sum() / (O ** 2).sum()))
    assert 1e-13 < err < 1e-6, err
    G.close()


def test_partition_handles_and_nccl_id():
    """A rank's handle covers its own elements; the NCCL id is made through
    the lazily loaded NCCL library; stepping without an exchange is refused."""
    import dgm_b200
    m = dgm_b200.meshgen.box(3, (2, 2, 2), 0.0, 2 * np.pi, 2)
    part = np.array([0, 0, 0, 0, 1, 1, 1, 1])
    R = dgm_b200.Domain.partition(m, dgm_b200.EULER3D, part, 2, 1)
    ne, ng, gl = R.partition_info()
    assert ne == 4 and ng == 4 and list(gl) == [4, 5, 6, 7]
    nid = dgm_b200.nccl_unique_id()
    assert len(nid) == 128 and any(nid)
    x, y, z = R.coordinates()
    with pytest.raises(dgm_b200.DgmxError):
        R.set_state(ics.taylor_green(x, y, z, Ma=0.1))


def _rank_run(rank, nranks, port, case, result):
    """One rank of a partitioned run: its own process and CUDA context on
    device 0, halo exchanges staged through the host over gloo (no kernel
    waits on another process)."""
    import datetime
    import os as _os
    import torch.distributed as dist
    import dgm_b200
    _os.environ["MASTER_ADDR"] = "127.0.0.1"
    _os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks, timeout=datetime.timedelta(seconds=60))
    phys, n, p, flux, inttype, dt, steps, vis, prec, hold = case
    m, rec, ic = _case_mesh(n, p, hold)
    ne = m.verts.shape[0]
    part = (np.arange(ne) * nranks) // ne
    D = dgm_b200.Domain.partition(m, phys, part, nranks, rank, flux=flux, inttype=inttype, vis=vis, precision=prec,
                                  boundaries=rec, bulk_hold=hold)
    D.set_exchange_host()
    nl, ng, gids = D.partition_info()
    x, y, z = D.coordinates()
    D.set_state(ic(x, y, z))
    D.advance(dt, steps)
    result[rank] = (gids.copy(), D.state())
    dist.barrier()
    dist.destroy_process_group()


def _case_mesh(n, p, walls):
    """Periodic box [0,2pi]^3 with the Taylor-Green state, or the channel:
    [0,2pi]^2 x [0,2] with isothermal walls at z = 0 and z = 2 and the
    wall-bounded shear flow."""
    import dgm_b200
    from tests.test_gpu_boundaries import channel_ic, wall_records
    if not walls:
        return dgm_b200.meshgen.box(3, n, 0.0, 2 * np.pi, p), None, lambda x, y, z: ics.taylor_green(x, y, z, Ma=0.1)
    m = dgm_b200.meshgen.box(3, n, (0.0, 0.0, 0.0), (2 * np.pi, 2 * np.pi, 2.0), p)
    return m, wall_records(n, BC_ISOTHERMAL_WALL, 1.0, 178.575), channel_ic


HOLD_CASES = [
    # name, n, p, flux, inttype, dt, steps, vis, nparts, kind, hold
    ("ns3d-walls-hold-lsrk14-2-slabs", (3, 2, 4), 3, "laxfriedrichs", 14, 0.001, 2, 0.02, 2, "slabs", True),
    ("ns3d-walls-hold-rk4-3-random", (2, 3, 4), 2, "laxfriedrichs", 4, 0.001, 2, 0.01, 3, "random", True),
    ("ns3d-walls-tvd3-2-random", (2, 2, 3), 3, "laxfriedrichs", 3, 0.001, 3, 0.02, 2, "random", False),
]


@pytest.mark.parametrize("case", HOLD_CASES, ids=[c[0] for c in HOLD_CASES])
def test_group_walls_and_hold_equal_single_domain(case):
    """Boundary sides and the channel's bulk-flow hold on an element
    partition: each part keeps its own wall sides, and the hold's means are
    taken over the whole mesh in global element order (every part's constant
    coefficients gathered after each stage), so the state equals the
    unpartitioned domain's bit for bit."""
    import dgm_b200
    _, n, p, flux, inttype, dt, steps, vis, nparts, kind, hold = case
    m, rec, ic = _case_mesh(n, p, True)
    ne = m.verts.shape[0]
    part = ((np.arange(ne) * nparts) // ne if kind == "slabs"
            else np.random.default_rng(11).permutation(np.arange(ne) % nparts))
    D = dgm_b200.Domain(m, 9, flux=flux, inttype=inttype, vis=vis, boundaries=rec, bulk_hold=hold)
    G = dgm_b200.Group(m, 9, part, flux=flux, inttype=inttype, vis=vis, boundaries=rec, bulk_hold=hold)
    x, y, z = D.coordinates()
    f = ic(x, y, z)
    D.set_state(f)
    G.set_state(f)
    D.advance(dt, steps)
    G.advance(dt, steps)
    S = D.state()
    assert np.array_equal(G.state(), S)
    assert not np.array_equal(S, f)
    G.close()


@pytest.mark.parametrize("case", [(8, (3, 2, 4), 3, "roe", 14, 0.002, 2, 0.0, 0, False),
                                  (9, (2, 2, 3), 2, "laxfriedrichs", 3, 0.002, 2, 0.02, 0, False),
                                  (8, (3, 2, 4), 3, "roe", 14, 0.002, 2, 0.0, 1, False),
                                  (9, (3, 2, 4), 3, "laxfriedrichs", 14, 0.001, 2, 0.02, 0, True)],
                         ids=["euler3d-lsrk14", "ns3d-tvd3", "euler3d-lsrk14-mixed", "ns3d-walls-hold-lsrk14"])
def test_two_process_ranks_equal_single_domain(case):
    """Two processes, each one rank of a partitioned domain, exchanging halos
    through the host: the gathered state equals the unpartitioned run (the
    mixed form's ranks gather the reference state's element integrals, and
    the bulk-flow hold's ranks every stage's constant coefficients, through
    the same transport)."""
    import socket
    import torch.multiprocessing as mp
    import dgm_b200
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    result = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank_run, args=(r, 2, port, case, result)) for r in range(2)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=300)
    for pr in procs:
        if pr.is_alive():
            pr.kill()
        assert pr.exitcode == 0
    phys, n, p, flux, inttype, dt, steps, vis, prec, hold = case
    m, rec, ic = _case_mesh(n, p, hold)
    D = dgm_b200.Domain(m, phys, flux=flux, inttype=inttype, vis=vis, precision=prec, boundaries=rec,
                        bulk_hold=hold)
    x, y, z = D.coordinates()
    D.set_state(ic(x, y, z))
    D.advance(dt, steps)
    S = D.state()
    qd = (p + 2) ** 3
    G = np.zeros_like(S).reshape(S.shape[0], -1, qd)
    for r in range(2):
        gids, loc = result[r]
        G[:, gids] = loc.reshape(S.shape[0], -1, qd)
    assert np.array_equal(G.reshape(S.shape), S)
