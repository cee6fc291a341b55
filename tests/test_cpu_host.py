"""CPU-only checks of the product's host side (no CUDA calls): the C ABI
library loads and exports every declared symbol, the 1-D tables agree with
the oracle, and the processed connectivity (masters, orientation
permutations) agrees with the oracle's restatement of Field::set_flip."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import oracle
from oracle import dgm_io

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lib():
    import dgm_b200
    return dgm_b200.lib()


def test_library_exports_every_declared_symbol():
    names = set()
    for h in sorted(glob.glob(os.path.join(ROOT, "include", "*.h"))):
        names |= set(re.findall(r"\b(dgmx_[a-z_]+)\s*\(", open(h).read()))
    L = _lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    assert len(names) >= 30


@pytest.mark.parametrize("L_,Q", [(2, 3), (4, 5), (5, 5), (5, 6), (8, 9), (8, 8)])
def test_tables_match_oracle(L_, Q):
    D = ctypes.POINTER(ctypes.c_double)
    G = Q - 1
    z, w = np.zeros(Q), np.zeros(Q)
    Dm, B, Bg = np.zeros((Q, Q)), np.zeros((L_, Q)), np.zeros((L_, G))
    a, b = np.zeros((G, Q)), np.zeros((Q, G))
    L = _lib()
    L.dgmx_tables.argtypes = [ctypes.c_int, ctypes.c_int] + [D] * 7
    assert L.dgmx_tables(L_, Q, *[x.ctypes.data_as(D) for x in (z, w, Dm, B, Bg, a, b)]) == 0
    t = oracle.tables(L_, Q, G)
    assert np.abs(z - t["z"]).max() < 1e-15
    assert np.abs(w - t["w"]).max() < 1e-15
    assert np.abs(Dm - t["D"]).max() < 1e-14 * np.abs(t["D"]).max()
    assert np.abs(B - t["B"]).max() < 1e-14
    assert np.abs(a - t["gl2g"]).max() < 1e-14
    assert np.abs(b - t["g2gl"]).max() < 1e-14
    # Legendre on Gauss points = GL2G interpolation of the GLL samples
    assert np.abs(Bg - B @ t["gl2g"].T).max() < 1e-14


def _links(mesh):
    import dgm_b200
    L = _lib()
    nf = 4 if mesh.dim == 2 else 6
    G = int(mesh.qorder[0]) - 1
    gf = G if mesh.dim == 2 else G * G
    verts = np.ascontiguousarray(mesh.verts, float)
    con = np.ascontiguousarray(mesh.con, np.int32)
    por = np.ascontiguousarray(mesh.porder, np.int32)
    qor = np.ascontiguousarray(mesh.qorder, np.int32)
    m = dgm_b200._Mesh(mesh.dim, verts.shape[0], verts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                       con.shape[0], con.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                       por.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                       qor.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    links = np.zeros((mesh.ne, nf, 4), np.int32)
    perm = np.zeros((mesh.ne, nf, gf), np.int32)
    L.dgmx_mesh_links.argtypes = [ctypes.POINTER(dgm_b200._Mesh), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int)]
    st = L.dgmx_mesh_links(ctypes.byref(m), links.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                           perm.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    assert st == 0
    return links, perm


def _oracle_pairs(mesh):
    """Point pairing implied by the oracle's side flags (master point
    side_map(q) <-> slave point q, src/Euler3d.cpp:601-612)."""
    P = oracle.Problem(mesh, oracle.EULER3D if mesh.dim == 3 else oracle.EULER2D)
    S = P.sides()
    G = int(mesh.qorder[0]) - 1
    n1, n2 = G, (G if mesh.dim == 3 else 1)

    def smap(flags, q):
        fa, fb, tr = flags
        if mesh.dim == 2:
            return (n1 - 1 - q) if fa else q
        il, jl = divmod(q, n2)
        if tr:
            j, i = il, jl
            if fa: j = n1 - 1 - j
            if fb: i = n2 - 1 - i
        else:
            i, j = il, jl
            if fa: i = n1 - 1 - i
            if fb: j = n2 - 1 - j
        return j + n2 * i
    pairs = {}
    for e in range(mesh.ne):
        for s in range(S.shape[1]):
            master, le, ls, fa, fb, tr = S[e, s]
            if master:
                for q in range(n1 * n2):
                    pairs[(e, s, smap((fa, fb, tr), q))] = (le, ls, q)
                    pairs[(le, ls, q)] = (e, s, smap((fa, fb, tr), q))
    return S, pairs


@pytest.mark.parametrize("which", ["box2d", "box3d", "rotated2d", "rotated3d", "vhex"])
def test_connectivity_matches_oracle(which):
    from tests.cases import load_golden, rotated_box
    if which == "box2d":
        mesh = dgm_io.box_mesh(2, (3, 4), -1, 1, 3)
    elif which == "box3d":
        mesh = dgm_io.box_mesh(3, (2, 3, 2), 0, 1, 2)
    elif which == "rotated2d":
        mesh = rotated_box(2, (3, 4), -1, 1, 3, seed=1)
    elif which == "rotated3d":
        mesh = rotated_box(3, (3, 3, 3), 0, 1, 3, seed=2)
    else:
        mesh, _, _ = load_golden("vhex")
        mesh = dgm_io.Mesh(3, mesh.verts, mesh.con, np.full(8, 3, np.int32), np.full(8, 5, np.int32))
    links, perm = _links(mesh)
    S, pairs = _oracle_pairs(mesh)
    ne, nfaces = links.shape[:2]
    for e in range(ne):
        for f in range(nfaces):
            assert links[e, f, 0] == S[e, f, 1] and links[e, f, 1] == S[e, f, 2]
            assert links[e, f, 2] == S[e, f, 0]
            for g in range(perm.shape[2]):
                le, ls, q = pairs[(e, f, g)]
                assert (le, ls) == (links[e, f, 0], links[e, f, 1])
                assert perm[e, f, g] == q


@pytest.mark.parametrize("world,layout,transport", [(1, "partition", "nccl"), (4, "partition", "nccl"),
                                                    (2, "partition", "host"), (8, "replicas", "nccl")])
def test_bench_arms_describe_the_same_workload(world, layout, transport):
    """Both arms of bench.py build their `config` with one function from the
    same arguments: at N > 1 the partitioned box grows with N (weak scaling)
    and the modal DOF counted are the whole job's."""
    import argparse
    import bench
    n, p, q = 32, 3, 5
    dof = 5 * n ** 3 * (p + 1) ** 3
    c = bench.config_dict(n, p, q, dof, world, layout, transport)
    assert c["workload"] == "euler3d_taylor_green_32^3_p3_roe_lsrk14"
    if world == 1:
        assert c["parallelism"] == "single device" and c["modal_dof"] == dof
    elif layout == "partition":
        assert c["modal_dof"] == dof * world
        assert c["mesh"].startswith(f"32x32x{32 * world} Hex")
        assert ("NCCL" in c["parallelism"]) == (transport == "nccl")
    else:
        assert c["modal_dof"] == dof and c["parallelism"].startswith("replicas")
    ns = argparse.Namespace(layout=layout, transport=transport)
    assert bench.config_dict(n, p, q, dof, world, ns.layout, ns.transport) == c
