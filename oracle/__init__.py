"""CPU FP64 oracle for DGM's DG residual + RK stage (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's ``cpu_baseline`` and
``--impl reference`` legs use this package.  The product (``dgm_b200``) never
imports it.  The numerics live in ``dgm_oracle.cpp`` (a line-by-line
restatement of the reference's algorithm, citations inside); this module only
loads that library and wraps it with ctypes.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libdgm_oracle.so")
_lib = None

# physics codes follow DGM's eqntype (src/ReoProblem.cpp:75-156)
EULER2D, NS2D, EULER3D, NS3D, SHALLOW = 1, 2, 8, 9, 30
FLUX = {"laxfriedrichs": 0, "roe": 1, "stegerwarming": 2, "vanleer": 3}


def build(force: bool = False) -> str:
    """Compile the oracle library with its Makefile (g++, no GPU needed)."""
    if force or not os.path.exists(_LIB_PATH) or (
            os.path.getmtime(_LIB_PATH) < os.path.getmtime(os.path.join(_HERE, "dgm_oracle.cpp"))):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        P, D, I = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
        L.ora_create.restype = P
        L.ora_create.argtypes = [ctypes.c_int, ctypes.c_int, D, I, I, ctypes.c_int, I,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double]
        L.ora_free.argtypes = [P]
        L.ora_ntot.restype = ctypes.c_long
        L.ora_ntot.argtypes = [P]
        L.ora_nmodes.restype = ctypes.c_long
        L.ora_nmodes.argtypes = [P]
        L.ora_nfields.argtypes = [P]
        L.ora_error.argtypes = [P]
        L.ora_set_threads.argtypes = [ctypes.c_int]
        L.ora_lsrk14_coefficients.argtypes = [D, D]
        L.ora_set_source.argtypes = [P, ctypes.c_void_p]
        L.ora_set_time.argtypes = [P, ctypes.c_double]
        L.ora_get_time.argtypes = [P]
        L.ora_get_time.restype = ctypes.c_double
        L.ora_set_source_pulse.argtypes = [P, ctypes.c_double, ctypes.c_double]
        L.ora_set_sw_balance.argtypes = [P, ctypes.c_int]
        L.ora_set_bc.argtypes = [P, ctypes.c_int, I, D]
        L.ora_set_hold_bulk.argtypes = [P, ctypes.c_int]
        L.ora_coords.argtypes = [P, D, D, D]
        L.ora_wj.argtypes = [P, D]
        L.ora_set_state.argtypes = [P, D]
        L.ora_get_state.argtypes = [P, D]
        L.ora_project.argtypes = [P, D]
        L.ora_forward.argtypes = [P, D, D]
        L.ora_backward.argtypes = [P, D, D]
        L.ora_rhs.argtypes = [P, D, D]
        L.ora_advance.argtypes = [P, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.ora_tables.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, D, D, D, D, D, D]
        L.ora_gauss.argtypes = [ctypes.c_int, D, D]
        L.ora_sides.argtypes = [P, I]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def tables(L: int, Q: int, G: int):
    """1-D tables (GLL z, w, D, orthonormal Legendre B, GL2G, G2GL)."""
    z, w = np.zeros(Q), np.zeros(Q)
    D, B = np.zeros((Q, Q)), np.zeros((L, Q))
    gl2g, g2gl = np.zeros((G, Q)), np.zeros((Q, G))
    lib().ora_tables(L, Q, G, _dp(z), _dp(w), _dp(D), _dp(B), _dp(gl2g), _dp(g2gl))
    return dict(z=z, w=w, D=D, B=B, gl2g=gl2g, g2gl=g2gl)


def gauss(np_: int):
    z, w = np.zeros(np_), np.zeros(np_)
    lib().ora_gauss(np_, _dp(z), _dp(w))
    return z, w


class Problem:
    """One DGM Domain restated on the CPU (Field layout: [field][element][Q^d])."""

    def __init__(self, mesh, physics: int, flux: str = "laxfriedrichs",
                 gamma: float = 1.4, vis: float = 0.0, Pr: float = 0.72):
        self.mesh = mesh
        self.dim = mesh.dim
        verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
        p = np.ascontiguousarray(mesh.porder, dtype=np.int32)
        q = np.ascontiguousarray(mesh.qorder, dtype=np.int32)
        con = np.ascontiguousarray(mesh.con, dtype=np.int32).reshape(-1)
        self.h = lib().ora_create(mesh.dim, mesh.ne, _dp(verts), _ip(p), _ip(q),
                                  len(mesh.con), _ip(con), physics, FLUX[flux.lower()],
                                  gamma, vis, Pr)
        if not self.h:
            raise RuntimeError("oracle: could not build the problem")
        self.nf = lib().ora_nfields(self.h)
        self.ntot = lib().ora_ntot(self.h)
        self.nmodes = lib().ora_nmodes(self.h)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().ora_free(h)
            self.h = None

    def coords(self):
        x, y, z = (np.zeros(self.ntot) for _ in range(3))
        lib().ora_coords(self.h, _dp(x), _dp(y), _dp(z))
        return x, y, z

    def wj(self):
        w = np.zeros(self.ntot)
        lib().ora_wj(self.h, _dp(w))
        return w

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.nf, self.ntot)
        lib().ora_set_state(self.h, _dp(U))

    def state(self):
        U = np.zeros((self.nf, self.ntot))
        lib().ora_get_state(self.h, _dp(U))
        return U

    def project(self, U):
        U = np.array(U, dtype=np.float64, order="C").reshape(self.nf, self.ntot)
        lib().ora_project(self.h, _dp(U))
        return U

    def forward(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.nf, self.ntot)
        Uh = np.zeros((self.nf, self.nmodes))
        lib().ora_forward(self.h, _dp(U), _dp(Uh))
        return Uh

    def backward(self, Uh):
        Uh = np.ascontiguousarray(Uh, dtype=np.float64).reshape(self.nf, self.nmodes)
        U = np.zeros((self.nf, self.ntot))
        lib().ora_backward(self.h, _dp(Uh), _dp(U))
        return U

    def rhs(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.nf, self.ntot)
        F = np.zeros_like(U)
        lib().ora_rhs(self.h, _dp(U), _dp(F))
        return F

    def advance(self, inttype: int, dt: float, nsteps: int) -> int:
        return lib().ora_advance(self.h, inttype, dt, nsteps)

    def set_bc(self, records):
        """Boundary sides: records (eid, sid, kind, params...) with up to five
        parameters; kind 1 slip wall (Euler), 2 isothermal wall (Tw, Eref;
        Navier-Stokes), 3 fixed state (the conserved values), 4 subsonic
        outflow (Mref; 2-D), 5 supersonic outflow (2-D)."""
        r = np.zeros((len(records), 8))
        for i, rec in enumerate(records):
            r[i, :len(rec)] = rec
        esk = np.ascontiguousarray(r[:, :3].astype(np.int32))
        par = np.ascontiguousarray(r[:, 3:8])
        if lib().ora_set_bc(self.h, len(r), _ip(esk), _dp(par)) != 0:
            raise ValueError("oracle: bad boundary record")

    def set_hold_bulk(self, on: bool):
        lib().ora_set_hold_bulk(self.h, 1 if on else 0)

    def set_sw_balance(self, on: bool):
        lib().ora_set_sw_balance(self.h, 1 if on else 0)

    def set_time(self, t: float):
        lib().ora_set_time(self.h, float(t))

    def time(self) -> float:
        return lib().ora_get_time(self.h)

    def set_source_pulse(self, t0: float, sigma_t: float):
        """Time factor exp(-(t - t0)^2 / (2 sigma_t^2)) on the source
        (Shallow::GaussianSource); sigma_t <= 0 removes it."""
        lib().ora_set_source_pulse(self.h, float(t0), float(sigma_t))

    def set_source(self, S):
        """Source field at the GLL points [nf][ntot] (2-D physics: F -= S
        before the projection); None removes it."""
        if S is None:
            lib().ora_set_source(self.h, None)
            return
        S = np.ascontiguousarray(S, dtype=np.float64).reshape(self.nf, self.ntot)
        self._S = S
        lib().ora_set_source(self.h, S.ctypes.data_as(ctypes.c_void_p))

    def error(self) -> int:
        return lib().ora_error(self.h)

    def sides(self):
        ns = 4 if self.dim == 2 else 6
        out = np.zeros((self.mesh.ne, ns, 6), dtype=np.int32)
        lib().ora_sides(self.h, _ip(out))
        return out


def set_threads(n: int):
    lib().ora_set_threads(int(n))


def lsrk14_coefficients():
    """LSRK14's 2N-storage coefficients (A, B) as the oracle steps with them
    (src/TimeInt.cpp:1870-1917)."""
    A, B = np.zeros(14), np.zeros(14)
    lib().ora_lsrk14_coefficients(A.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  B.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return A, B
