"""Element partitions on the host: the plan's ghost slots and exchange lists
(dgmx_partition_plan), and the halo exchange protocol run between two gloo
ranks on the CPU with the plan's own lists (pack by the send list, one
message per peer, unpack by the receive list)."""
import os
import socket

import numpy as np
import pytest

NFACE = 6
BLK = 3


def _mesh(n=(4, 3, 2), p=2):
    import dgm_b200
    return dgm_b200.meshgen.box(3, n, 0.0, 1.0, p)


def _parts(ne, nranks, kind):
    if kind == "slabs":
        return (np.arange(ne) * nranks) // ne
    return np.random.default_rng(11).integers(0, nranks, ne)


def _block(e, f):
    """The trace block of global face (e, f): values the test can recompute."""
    return np.array([1000.0 * e + 10.0 * f + k for k in range(BLK)])


@pytest.mark.parametrize("nranks,kind", [(2, "slabs"), (3, "slabs"), (4, "random")])
def test_plan_lists_pair_up(nranks, kind):
    import dgm_b200
    m = _mesh()
    ne = m.verts.shape[0]
    part = _parts(ne, nranks, kind)
    plans = [dgm_b200.partition_plan(m, part, nranks, r) for r in range(nranks)]
    links = np.zeros((ne, NFACE, 4), np.int32)
    perm = np.zeros((ne, NFACE, 16), np.int32)
    dgm_b200.lib().dgmx_mesh_links(_struct(m), links.ctypes.data_as(_ip()), perm.ctypes.data_as(_ip()))
    for r, pl in enumerate(plans):
        assert list(pl["global_of_local"]) == [e for e in range(ne) if part[e] == r]
        # every remote neighbour of a local face is a ghost
        need = sorted({int(links[e, f, 0]) for e in pl["global_of_local"] for f in range(NFACE)
                       if part[links[e, f, 0]] != r})
        assert list(pl["global_of_ghost"]) == need
        off = np.concatenate([[0], np.cumsum(pl["peer_counts"])])
        for q in range(nranks):
            other = plans[q]
            oq = np.concatenate([[0], np.cumsum(other["peer_counts"])])
            assert pl["peer_counts"][q] == other["peer_counts"][r]
            sent = [(int(pl["global_of_local"][b // NFACE]), b % NFACE) for b in pl["send"][off[q]:off[q + 1]]]
            got = [(int(other["global_of_ghost"][b // NFACE - len(other["global_of_local"])]), b % NFACE)
                   for b in other["recv"][oq[r]:oq[r + 1]]]
            assert sent == got            # same blocks, same order, no metadata exchanged
            assert sent == sorted(sent)


def _struct(m):
    import dgm_b200
    st, keep = dgm_b200._mesh_struct(m)
    _struct.keep = keep
    import ctypes
    return ctypes.byref(st)


def _ip():
    import ctypes
    return ctypes.POINTER(ctypes.c_int)


def _rank_main(rank, nranks, port, part, result):
    import torch.distributed as dist
    import dgm_b200
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks)
    import torch
    m = _mesh()
    pl = dgm_b200.partition_plan(m, part, nranks, rank)
    nloc, ngh = len(pl["global_of_local"]), len(pl["global_of_ghost"])
    T = np.full((nloc + ngh, NFACE, BLK), np.nan)
    for i, e in enumerate(pl["global_of_local"]):
        for f in range(NFACE):
            T[i, f] = _block(int(e), f)
    off = np.concatenate([[0], np.cumsum(pl["peer_counts"])])
    flat = T.reshape(-1, BLK)
    sbuf = flat[pl["send"]].copy()
    rbuf = np.zeros_like(sbuf)
    reqs = []
    for q in range(nranks):
        if q == rank or not pl["peer_counts"][q]:
            continue
        a, b = off[q], off[q + 1]
        reqs.append(dist.isend(torch.from_numpy(sbuf[a:b].copy()), q))
        rt = torch.zeros((b - a, BLK), dtype=torch.float64)
        reqs.append((dist.irecv(rt, q), rt, a, b))
    for r_ in reqs:
        if isinstance(r_, tuple):
            r_[0].wait()
            rbuf[r_[2]:r_[3]] = r_[1].numpy()
        else:
            r_.wait()
    flat[pl["recv"]] = rbuf
    # every local face whose neighbour is remote now reads the neighbour's block
    links = np.zeros((m.verts.shape[0], NFACE, 4), np.int32)
    perm = np.zeros((m.verts.shape[0], NFACE, 16), np.int32)
    dgm_b200.lib().dgmx_mesh_links(_struct(m), links.ctypes.data_as(_ip()), perm.ctypes.data_as(_ip()))
    slot = {int(g): nloc + i for i, g in enumerate(pl["global_of_ghost"])}
    ok = True
    for e in pl["global_of_local"]:
        for f in range(NFACE):
            le, lf = int(links[e, f, 0]), int(links[e, f, 1])
            if part[le] != rank:
                ok &= bool(np.array_equal(T[slot[le], lf], _block(le, lf)))
    result[rank] = int(ok)
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["slabs", "random"])
def test_halo_exchange_between_gloo_ranks(kind):
    import torch.multiprocessing as mp
    nranks = 2
    m = _mesh()
    part = _parts(m.verts.shape[0], nranks, kind)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    result = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank_main, args=(r, nranks, port, part, result)) for r in range(nranks)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    assert dict(result) == {0: 1, 1: 1}


def test_nccl_resolution_keeps_torch_importable():
    """The engine resolves NCCL lazily; making an id before the host's own
    PyTorch import must not leave a different libnccl.so.2 in the process."""
    import subprocess
    import sys
    code = ("import sys; sys.path.insert(0, %r); import dgm_b200; i = dgm_b200.nccl_unique_id(); "
            "import torch; assert len(i) == 128" % os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
