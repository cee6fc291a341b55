"""Periodic box meshes in DGM's mesh/connectivity layout (host setup).

Element numbering, vertex order and periodic links follow DGM's box
generator (src/Mesh.cpp:472-490 for Quads, the Hex analogue at :879-884):
element id = i + nx*(j + ny*k), counter-clockwise vertices, one connectivity
record per element side in side order.  Vectorised with numpy so the 32^3 and
larger meshes of the benchmark configurations build in milliseconds.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass
class Mesh:
    dim: int
    verts: np.ndarray      # (ne, 4|8, 3)
    con: np.ndarray        # (ncon, 4) eid, side, link eid, link side
    porder: np.ndarray     # (ne,)
    qorder: np.ndarray     # (ne,)

    @property
    def ne(self) -> int:
        return int(self.verts.shape[0])


def box(dim: int, n, lo, hi, p: int, q: int = 0) -> Mesh:
    n = np.broadcast_to(np.asarray(n, dtype=np.int64), (dim,))
    lo = np.broadcast_to(np.asarray(lo, dtype=np.float64), (dim,))
    hi = np.broadcast_to(np.asarray(hi, dtype=np.float64), (dim,))
    h = (hi - lo) / n
    if dim == 2:
        nx, ny = (int(v) for v in n)
        j, i = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        i, j = i.ravel(), j.ravel()
        e = i + j * nx
        corner = np.array([(0, 0), (1, 0), (1, 1), (0, 1)])
        verts = np.zeros((e.size, 4, 3))
        verts[:, :, 0] = lo[0] + (i[:, None] + corner[None, :, 0]) * h[0]
        verts[:, :, 1] = lo[1] + (j[:, None] + corner[None, :, 1]) * h[1]
        idx = lambda a, b: (a % nx) + (b % ny) * nx
        nb = [idx(i, j - 1), idx(i + 1, j), idx(i, j + 1), idx(i - 1, j)]
        opp = [2, 3, 0, 1]
        con = np.stack([np.stack([e, np.full_like(e, s), nb[s], np.full_like(e, opp[s])], 1) for s in range(4)], 1)
    else:
        nx, ny, nz = (int(v) for v in n)
        k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        i, j, k = i.ravel(), j.ravel(), k.ravel()
        e = i + nx * (j + ny * k)
        corner = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
                           (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)])
        verts = np.zeros((e.size, 8, 3))
        for c, ax in enumerate((i, j, k)):
            verts[:, :, c] = lo[c] + (ax[:, None] + corner[None, :, c]) * h[c]
        idx = lambda a, b, c: (a % nx) + nx * ((b % ny) + ny * (c % nz))
        # Hex sides: 0 z-, 1 y-, 2 x+, 3 y+, 4 x-, 5 z+ (src/Hex.cpp:68-69)
        nb = [idx(i, j, k - 1), idx(i, j - 1, k), idx(i + 1, j, k), idx(i, j + 1, k), idx(i - 1, j, k),
              idx(i, j, k + 1)]
        opp = [5, 3, 4, 1, 2, 0]
        con = np.stack([np.stack([e, np.full_like(e, s), nb[s], np.full_like(e, opp[s])], 1) for s in range(6)], 1)
    con = con.reshape(-1, 4).astype(np.int32)
    ne = verts.shape[0]
    return Mesh(dim, verts, con, np.full(ne, p, np.int32), np.full(ne, q if q else p + 2, np.int32))


def gll_coordinates(mesh: Mesh, z):
    """GLL point coordinates in Field layout for an affine box mesh (host helper)."""
    Q = z.size
    a0, a1 = 0.5 * (1 - z), 0.5 * (1 + z)
    V = mesh.verts
    if mesh.dim == 2:
        w = [np.einsum("i,j->ij", a0, a0), np.einsum("i,j->ij", a1, a0),
             np.einsum("i,j->ij", a1, a1), np.einsum("i,j->ij", a0, a1)]
        out = [sum(V[:, v, c][:, None, None] * w[v][None] for v in range(4)).reshape(-1) for c in range(2)]
        return out[0], out[1], np.zeros_like(out[0])
    sel = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)]
    ab = (a0, a1)
    w = [np.einsum("i,j,k->ijk", ab[s[0]], ab[s[1]], ab[s[2]]) for s in sel]
    return tuple(sum(V[:, v, c][:, None, None, None] * w[v][None] for v in range(8)).reshape(-1) for c in range(3))
