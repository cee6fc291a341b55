"""dgm_b200: B200-native DG residual + RK-stage engine with DGM's Domain interface.

The compute path is libdgmx.so (hand-written sm_100a CUDA kernels behind the
C ABI in include/dgmx.h).  This module is the host-side mirror of DGM's
Domain/TimeInt interface over that ABI: ``Domain.time_derivative(U, F)``
(src/Domain.hpp:243), ``Domain.advance(dt, nsteps)`` (TimeInt::advance,
src/TimeInt.hpp:177-181), ``Domain.set_ic``-style state setting with
projection, and restart-layout modal output.  There is no CPU fallback: if
the library or a CUDA device is missing, construction raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import meshgen  # noqa: F401

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdgmx.so")
_lib = None

EULER2D, NS2D, EULER3D, NS3D, SHALLOW = 1, 2, 8, 9, 30
TVD3, RK4, LSRK14 = 3, 4, 14
FP64, MIXED = 0, 1
FLUX = {"laxfriedrichs": 0, "lf": 0, "roe": 1, "stegerwarming": 2, "vanleer": 3}
STATUS = {0: "ok", 1: "argument", 2: "unsupported", 3: "cuda", 4: "non-physical", 5: "io", 6: "memory"}


class DgmxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"dgmx {STATUS.get(code, code)} error: {msg}")
        self.code = code


class NonPhysicalState(DgmxError):
    pass


class _Mesh(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("ne", ctypes.c_int), ("verts", ctypes.POINTER(ctypes.c_double)),
                ("ncon", ctypes.c_int), ("con", ctypes.POINTER(ctypes.c_int)),
                ("porder", ctypes.POINTER(ctypes.c_int)), ("qorder", ctypes.POINTER(ctypes.c_int))]


class _Params(ctypes.Structure):
    _fields_ = [("physics", ctypes.c_int), ("flux", ctypes.c_int), ("inttype", ctypes.c_int),
                ("precision", ctypes.c_int), ("sw_balance", ctypes.c_int), ("device", ctypes.c_int),
                ("gamma", ctypes.c_double), ("vis", ctypes.c_double), ("Pr", ctypes.c_double)]


def lib():
    """Load libdgmx.so (built by __graft_entry__.build / dgm_b200.build)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise DgmxError(3, f"{LIB_PATH} is missing: run python -m dgm_b200.build")
        L = ctypes.CDLL(LIB_PATH)
        P, D, I = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
        L.dgmx_create.argtypes = [ctypes.POINTER(_Mesh), ctypes.POINTER(_Params), ctypes.POINTER(P)]
        L.dgmx_create_from_files.argtypes = [ctypes.c_char_p, ctypes.POINTER(_Params), ctypes.POINTER(P)]
        L.dgmx_destroy.argtypes = [P]
        L.dgmx_sizes.argtypes = [P, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(ctypes.c_long),
                                 ctypes.POINTER(ctypes.c_long)]
        L.dgmx_coordinates.argtypes = [P, D, D, D]
        for f in ("dgmx_set_state", "dgmx_get_state", "dgmx_get_modes", "dgmx_integrals"):
            getattr(L, f).argtypes = [P, D]
        for f in ("dgmx_set_state_device", "dgmx_get_state_device"):
            getattr(L, f).argtypes = [P, ctypes.c_void_p]
        L.dgmx_time_derivative.argtypes = [P, D, D]
        L.dgmx_time_derivative_device.argtypes = [P, ctypes.c_void_p, ctypes.c_void_p]
        L.dgmx_advance.argtypes = [P, ctypes.c_double, I]
        L.dgmx_advance_async.argtypes = [P, ctypes.c_double, I]
        L.dgmx_sync.argtypes = [P]
        L.dgmx_last_error.argtypes = [P]
        L.dgmx_last_error.restype = ctypes.c_char_p
        L.dgmx_launch_count.argtypes = [P]
        L.dgmx_launch_count.restype = ctypes.c_long
        L.dgmx_kernel_list.argtypes = [ctypes.POINTER(ctypes.c_int), I]
        L.dgmx_stream.argtypes = [P]
        L.dgmx_stream.restype = ctypes.c_void_p
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def fma_peak(fp64: bool = True, device: int = 0, reps: int = 5) -> float:
    """Measured FMA throughput of the GPU in TFLOP/s (FP64 or FP32)."""
    f = lib().dgmx_measure_fma_peak
    f.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    t = ctypes.c_double()
    st = f(int(device), 1 if fp64 else 0, int(reps), ctypes.byref(t))
    if st != 0:
        raise DgmxError(st, "FMA peak measurement failed")
    return t.value


def kernel_list():
    """Compiled instantiations: rows of (physics, L, Q, elements/CTA, threads, smem bytes, min CTAs/SM)."""
    n = 4096
    buf = (ctypes.c_int * (7 * n))()
    k = lib().dgmx_kernel_list(buf, n)
    return np.frombuffer(buf, dtype=np.int32)[: 7 * k].reshape(k, 7).copy()


# boundary kinds (include/dgmx.h)
BC_SLIP_WALL, BC_ISOTHERMAL_WALL, BC_STATE, BC_SUBSONIC_OUTFLOW, BC_SUPERSONIC_OUTFLOW = 1, 2, 3, 4, 5


def _bc_arrays(boundaries):
    """(count, sides [n][3] int32, parameters [n][5]) of boundary records
    (element, side, kind, up to five parameters); count 0 for None."""
    recs = list(boundaries) if boundaries is not None else []
    r = np.zeros((max(len(recs), 1), 8))
    for i, rec in enumerate(recs):
        r[i, :len(rec)] = rec
    return (len(recs), np.ascontiguousarray(r[:, :3].astype(np.int32)), np.ascontiguousarray(r[:, 3:8]))


class Domain:
    """One DGM Domain on one GPU (Field layout [field][element][Q^d])."""

    def __init__(self, mesh, physics: int, flux: str = "laxfriedrichs", inttype: int = LSRK14,
                 gamma: float = 1.4, vis: float = 0.0, Pr: float = 0.72, sw_balance: bool = True,
                 device: int = 0, precision: int = 0, boundaries=None, bulk_hold: bool = False):
        """boundaries: optional (element, side, kind, params...) records
        with up to five parameters: BC_SLIP_WALL (Euler), BC_ISOTHERMAL_WALL
        (Tw, Eref; Navier-Stokes), BC_STATE (the conserved values),
        BC_SUBSONIC_OUTFLOW (Mref; 2-D), BC_SUPERSONIC_OUTFLOW (2-D);
        bulk_hold: the channel's bulk-flow hold (Navier-Stokes 3-D)."""
        self._keep = []
        verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
        con = np.ascontiguousarray(mesh.con, dtype=np.int32)
        por = np.ascontiguousarray(mesh.porder, dtype=np.int32)
        qor = np.ascontiguousarray(mesh.qorder, dtype=np.int32)
        self._keep += [verts, con, por, qor]
        m = _Mesh(int(mesh.dim), int(verts.shape[0]), _dp(verts), int(con.shape[0]),
                  con.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                  por.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                  qor.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        p = _Params(physics, FLUX[flux.lower()], inttype, precision, 1 if sw_balance else 0, device,
                    gamma, vis, Pr)
        h = ctypes.c_void_p()
        if boundaries is None:
            st = lib().dgmx_create(ctypes.byref(m), ctypes.byref(p), ctypes.byref(h))
        else:
            r = np.zeros((len(boundaries), 8))
            for i, rec in enumerate(boundaries):
                r[i, :len(rec)] = rec
            sides = np.ascontiguousarray(r[:, :3].astype(np.int32))
            par = np.ascontiguousarray(r[:, 3:8])
            f = lib().dgmx_create_with_boundaries
            f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                          ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
            st = f(ctypes.byref(m), ctypes.byref(p), len(r), sides.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                   _dp(par), ctypes.byref(h))
        if st != 0:
            raise DgmxError(st, lib().dgmx_last_error(None).decode())
        self._init(h, mesh.dim)
        if bulk_hold:
            self.set_bulk_hold(True)

    @classmethod
    def partition(cls, mesh, physics: int, part, nranks: int, rank: int, flux: str = "laxfriedrichs",
                  inttype: int = LSRK14, gamma: float = 1.4, vis: float = 0.0, Pr: float = 0.72,
                  sw_balance: bool = True, device: int = 0, precision: int = FP64, boundaries=None,
                  bulk_hold: bool = False):
        """The rank's part of an element partition (part[e] = owning rank);
        its arrays cover its own elements in increasing global order.  Call
        set_exchange_nccl (or set_exchange_host) on every rank before
        setting the state: with precision=MIXED, set_state gathers every
        rank's element integrals for the common reference state.
        boundaries: the records of the constructor, global element ids;
        bulk_hold: the channel's hold with its means over the whole mesh."""
        m, keep = _mesh_struct(mesh)
        part = np.ascontiguousarray(part, dtype=np.int32)
        p = _Params(physics, FLUX[flux.lower()], inttype, precision, 1 if sw_balance else 0, device, gamma, vis, Pr)
        h = ctypes.c_void_p()
        nbc, sides, par = _bc_arrays(boundaries)
        f = lib().dgmx_create_partition_with_boundaries
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
                      ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
        st = f(ctypes.byref(m), ctypes.byref(p), part.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), int(nranks),
               int(rank), nbc, sides.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(par), ctypes.byref(h))
        if st != 0:
            raise DgmxError(st, lib().dgmx_last_error(None).decode())
        self = cls.__new__(cls)
        self._keep = keep + [part, sides, par]
        self._init(h, mesh.dim)
        if bulk_hold:
            self.set_bulk_hold(True)
        return self

    def set_exchange_nccl(self, nccl_id: bytes):
        """NCCL communicator for the halo exchange (collective over the ranks)."""
        _nccl_first()
        f = lib().dgmx_set_exchange_nccl
        f.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        self._check(f(self.h, bytes(nccl_id)))

    def set_exchange_host(self, group=None):
        """Host-staged halo exchange through torch.distributed (any backend
        with point-to-point sends, e.g. gloo): at every exchange the packed
        face blocks come to the host, go to the peers and back.  Collective
        over the ranks; steps are then not captured into graphs."""
        import torch
        import torch.distributed as dist
        FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                              ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int),
                              ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int)
        me = dist.get_rank(group)

        def transport(ctx, send, recv, counts, offsets, blk, nranks):
            try:
                total = sum(counts[q] for q in range(nranks)) * blk
                if total == 0:
                    return 0
                sa = np.ctypeslib.as_array(send, shape=(total,))
                ra = np.ctypeslib.as_array(recv, shape=(total,))
                sends, recvs = [], []
                for q in range(nranks):
                    n = counts[q] * blk
                    if q == me or n == 0:
                        continue
                    o = offsets[q] * blk
                    sends.append(dist.isend(torch.from_numpy(sa[o:o + n].copy()), q, group=group))
                    buf = torch.empty(n, dtype=torch.float64)
                    recvs.append((dist.irecv(buf, q, group=group), buf, o, n))
                for r in sends:
                    r.wait()
                for r, buf, o, n in recvs:
                    r.wait()
                    ra[o:o + n] = buf.numpy()
                return 0
            except Exception:
                return 1

        self._xfn = FN(transport)   # kept alive with the handle
        f = lib().dgmx_set_exchange_host
        f.argtypes = [ctypes.c_void_p, FN, ctypes.c_void_p]
        self._check(f(self.h, self._xfn, None))

    def partition_info(self):
        """(local element count, ghost slots, global id of every local element)."""
        ne, ng = ctypes.c_int(), ctypes.c_int()
        f = lib().dgmx_partition_info
        f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                      ctypes.POINTER(ctypes.c_int)]
        self._check(f(self.h, ctypes.byref(ne), ctypes.byref(ng), None))
        g = np.zeros(ne.value, dtype=np.int32)
        self._check(f(self.h, None, None, g.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return ne.value, ng.value, g

    @classmethod
    def from_files(cls, root: str, inttype: int = TVD3, physics: int = EULER3D, device: int = 0):
        """Domain from DGM input files root.inp/.msh/.con/.ord."""
        p = _Params(physics, 0, inttype, 0, 1, device, 1.4, 0.0, 0.72)
        h = ctypes.c_void_p()
        st = lib().dgmx_create_from_files(root.encode(), ctypes.byref(p), ctypes.byref(h))
        if st != 0:
            raise DgmxError(st, lib().dgmx_last_error(None).decode())
        self = cls.__new__(cls)
        self._keep = []
        nf, nq, nm = ctypes.c_long(), ctypes.c_long(), ctypes.c_long()
        lib().dgmx_sizes(h, ctypes.byref(nf), ctypes.byref(nq), ctypes.byref(nm))
        self._init(h, None)
        return self

    def _init(self, h, dim):
        self.h = h
        nf, nq, nm = ctypes.c_long(), ctypes.c_long(), ctypes.c_long()
        lib().dgmx_sizes(h, ctypes.byref(nf), ctypes.byref(nq), ctypes.byref(nm))
        self.nf, self.nq, self.nm = nf.value, nq.value, nm.value
        self.dim = dim

    def close(self):
        if getattr(self, "h", None):
            lib().dgmx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            msg = lib().dgmx_last_error(self.h).decode()
            raise (NonPhysicalState if st == 4 else DgmxError)(st, msg)

    # --- data movement -------------------------------------------------
    def coordinates(self):
        x, y, z = (np.zeros(self.nq) for _ in range(3))
        self._check(lib().dgmx_coordinates(self.h, _dp(x), _dp(y), _dp(z)))
        return x, y, z

    def set_state(self, U):
        """Set U (GLL values, Field layout) and project it (set_ic + project)."""
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.nf, self.nq)
        self._check(lib().dgmx_set_state(self.h, _dp(U)))

    def state(self):
        U = np.zeros((self.nf, self.nq))
        self._check(lib().dgmx_get_state(self.h, _dp(U)))
        return U

    def _check_host_buffer(self, U):
        """A host array the engine copies the whole state into or out of:
        float64, C-contiguous, nf * nq values (anything else would let the
        copy run past the array)."""
        if not isinstance(U, np.ndarray):
            raise ValueError("state buffer must be a numpy array")
        if U.dtype != np.float64:
            raise ValueError(f"state buffer must be float64, got {U.dtype}")
        if not U.flags.c_contiguous:
            raise ValueError("state buffer must be C-contiguous")
        if U.size != self.nf * self.nq:
            raise ValueError(f"state buffer holds {U.size} values, the state has {self.nf * self.nq}")

    def state_into(self, U):
        """get_state into a caller array (page-locked arrays are written by DMA)."""
        self._check_host_buffer(U)
        self._check(lib().dgmx_get_state(self.h, _dp(U)))
        return U

    def set_state_async(self, U):
        """set_state without the host wait; U: a page-locked (pinned)
        float64 array in the Field layout, left untouched until sync()."""
        f = lib().dgmx_set_state_async
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._check_host_buffer(U)
        self._check(f(self.h, U.ctypes.data_as(ctypes.c_void_p)))

    def state_async(self, U):
        """get_state into a page-locked array without the host wait; U holds
        the state once sync() returns."""
        f = lib().dgmx_get_state_async
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._check_host_buffer(U)
        self._check(f(self.h, U.ctypes.data_as(ctypes.c_void_p)))
        return U

    def modes(self):
        """Restart-layout modal coefficients [field][element][L^d]."""
        Uh = np.zeros((self.nf, self.nm))
        self._check(lib().dgmx_get_modes(self.h, _dp(Uh)))
        return Uh

    def set_state_device(self, ptr: int):
        self._check(lib().dgmx_set_state_device(self.h, ctypes.c_void_p(ptr)))

    def state_device(self, ptr: int):
        self._check(lib().dgmx_get_state_device(self.h, ctypes.c_void_p(ptr)))

    # --- the hot path --------------------------------------------------
    def time_derivative(self, U, F=None):
        """Domain::time_derivative: returns F = -dU/dt (projected) at GLL points."""
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.nf, self.nq)
        if F is None:
            F = np.zeros_like(U)
        self._check(lib().dgmx_time_derivative(self.h, _dp(U), _dp(F)))
        return F

    def time_derivative_device(self, U_ptr: int, F_ptr: int):
        self._check(lib().dgmx_time_derivative_device(self.h, ctypes.c_void_p(U_ptr), ctypes.c_void_p(F_ptr)))

    def advance(self, dt: float, nsteps: int = 1):
        """TimeInt::advance repeated nsteps times (device resident)."""
        self._check(lib().dgmx_advance(self.h, float(dt), int(nsteps)))

    def advance_async(self, dt: float, nsteps: int = 1):
        self._check(lib().dgmx_advance_async(self.h, float(dt), int(nsteps)))

    def sync(self):
        self._check(lib().dgmx_sync(self.h))

    def integrals(self):
        out = np.zeros(self.nf)
        self._check(lib().dgmx_integrals(self.h, _dp(out)))
        return out

    def launch_count(self) -> int:
        return lib().dgmx_launch_count(self.h)

    def autotune(self, reps: int = 20):
        """Pick the fastest compiled tile variant on this mesh; returns
        (rows of (epb, minb, threads, us per launch), chosen index)."""
        L = lib()
        f = L.dgmx_autotune
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int,
                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        rows = np.zeros((64, 4))
        nv, ch = ctypes.c_int(), ctypes.c_int()
        self._check(f(self.h, int(reps), _dp(rows), 64, ctypes.byref(nv), ctypes.byref(ch)))
        return rows[: nv.value].copy(), ch.value

    def set_source(self, S):
        """Time-independent source of the 2-D physics: F -= S at the GLL
        points before the projection (FileSource / ConstSource).  S: GLL
        values (Field layout, as set_state), nf constants (ConstSource), or
        None to remove it.  3-D domains raise: the reference applies no
        source there."""
        f = lib().dgmx_set_source
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        if S is None:
            self._check(f(self.h, None))
            return
        S = np.asarray(S, dtype=np.float64)
        if S.ndim == 1 and S.size == self.nf:
            S = np.repeat(S[:, None], self.nq, axis=1)
        S = np.ascontiguousarray(S).reshape(self.nf, self.nq)
        self._check(f(self.h, S.ctypes.data_as(ctypes.c_void_p)))

    def set_time(self, t: float):
        """Domain::t (advance adds dt per step)."""
        f = lib().dgmx_set_time
        f.argtypes = [ctypes.c_void_p, ctypes.c_double]
        self._check(f(self.h, float(t)))

    def time(self) -> float:
        f = lib().dgmx_get_time
        f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        t = ctypes.c_double()
        self._check(f(self.h, ctypes.byref(t)))
        return t.value

    def set_source_pulse(self, t0: float, sigma_t: float):
        """Time factor exp(-(t - t0)^2 / (2 sigma_t^2)) on the source, the form
        of Shallow::GaussianSource; sigma_t <= 0 removes it."""
        f = lib().dgmx_set_source_pulse
        f.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        self._check(f(self.h, float(t0), float(sigma_t)))

    def set_bulk_hold(self, on: bool):
        """Channel::holdBulkMassFlow after every projected RHS (Navier-Stokes 3-D)."""
        f = lib().dgmx_set_bulk_hold
        f.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self._check(f(self.h, 1 if on else 0))

    def set_variant(self, index: int):
        """Use compiled tile variant `index`; returns (variant count, kind): kind 0 is a
        CTA tile, 2 the prefetching persistent kernel."""
        f = lib().dgmx_set_variant
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        n, w = ctypes.c_int(), ctypes.c_int()
        self._check(f(self.h, int(index), ctypes.byref(n), ctypes.byref(w)))
        return n.value, int(w.value)

    def set_tensor_contractions(self, on: bool):
        """Navier-Stokes 3-D, p >= 5, FP32 viscous form: 3xTF32 tensor-core
        contractions in the viscous kernels (dgmx_set_tensor_contractions)."""
        f = lib().dgmx_set_tensor_contractions
        f.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self._check(f(self.h, 1 if on else 0))

    def set_wait_limit(self, tries: int):
        """Fault injection for tests: bound the prefetching stage kernel's
        first wait per tile to `tries` (0: every wait runs out, the call
        fails with DGMX_ERR_CUDA and the context stays usable); a negative
        value restores the default bound."""
        f = lib().dgmx_set_wait_limit
        f.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self._check(f(self.h, int(tries)))

    def variant_count(self) -> int:
        f = lib().dgmx_set_variant
        f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        n, w = ctypes.c_int(), ctypes.c_int()
        f(self.h, -1, ctypes.byref(n), ctypes.byref(w))
        return n.value

    # --- restart files (DGM format) -------------------------------------
    def set_modes(self, Uh):
        """Set the state from restart-layout modal coefficients [field][element][L^d]."""
        Uh = np.ascontiguousarray(Uh, dtype=np.float64).reshape(self.nf, self.nm)
        f = lib().dgmx_set_modes
        f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        self._check(f(self.h, _dp(Uh)))

    def write_restart(self, path: str, step: int = 0, t: float = 0.0, dt: float = 0.0):
        f = lib().dgmx_write_restart
        f.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        self._check(f(self.h, path.encode(), int(step), float(t), float(dt)))

    def read_restart(self, path: str):
        """Load a restart file into the state; returns (step, time)."""
        f = lib().dgmx_read_restart
        f.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
        step, t = ctypes.c_int(), ctypes.c_double()
        self._check(f(self.h, path.encode(), ctypes.byref(step), ctypes.byref(t)))
        return step.value, t.value

    def stream(self) -> int:
        """The handle's cudaStream_t as an integer (for torch.cuda.ExternalStream)."""
        return lib().dgmx_stream(self.h) or 0


# ---- restart files and Domain::diff (host only, no GPU needed) -----------
def _restart_err():
    f = lib().dgmx_restart_last_error
    f.restype = ctypes.c_char_p
    return f().decode()


def restart_write(path: str, physics: int, modes, step: int = 0, t: float = 0.0, dt: float = 0.0,
                  vis: float = 0.0):
    """Write modes [field][element][nmodes] as a DGM restart file."""
    modes = np.ascontiguousarray(modes, dtype=np.float64)
    nf, ne, nm = modes.shape
    f = lib().dgmx_restart_write
    f.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                  ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]
    st = f(path.encode(), int(physics), ne, nm, int(step), float(t), float(dt), float(vis), _dp(modes))
    if st != 0:
        raise DgmxError(st, _restart_err())


def restart_info(path: str) -> dict:
    f = lib().dgmx_restart_info
    I, D = ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
    f.argtypes = [ctypes.c_char_p, I, I, I, I, D, D, D]
    ne, nsd, lmax, step = (ctypes.c_int() for _ in range(4))
    t, dt, vis = (ctypes.c_double() for _ in range(3))
    st = f(path.encode(), ctypes.byref(ne), ctypes.byref(nsd), ctypes.byref(lmax), ctypes.byref(step),
           ctypes.byref(t), ctypes.byref(dt), ctypes.byref(vis))
    if st != 0:
        raise DgmxError(st, _restart_err())
    return dict(ne=ne.value, nsd=nsd.value, lmax=lmax.value, step=step.value, t=t.value, dt=dt.value,
                vis=vis.value)


def restart_read(path: str, nf: int):
    """(per-element mode counts, list of per-field coefficient arrays, header info)."""
    info = restart_info(path)
    ne = info["ne"]
    cap = nf * ne * info["lmax"]
    nmodes = np.zeros(ne, dtype=np.int32)
    modes = np.zeros(cap)
    f = lib().dgmx_restart_read
    f.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                  ctypes.POINTER(ctypes.c_double), ctypes.c_longlong]
    st = f(path.encode(), nf, ne, nmodes.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(modes), cap)
    if st != 0:
        raise DgmxError(st, _restart_err())
    tot = int(nmodes.sum())
    return nmodes, [modes[k * tot:(k + 1) * tot].copy() for k in range(nf)], info


def restart_diff(mesh, physics: int, rst1: str, rst2: str, aeps: float = -1.0, reps: float = -1.0):
    """Domain::diff of two restart files on `mesh`: (status bits, norms[nf][6])."""
    verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
    con = np.ascontiguousarray(mesh.con, dtype=np.int32)
    por = np.ascontiguousarray(mesh.porder, dtype=np.int32)
    qor = np.ascontiguousarray(mesh.qorder, dtype=np.int32)
    m = _Mesh(int(mesh.dim), int(verts.shape[0]), _dp(verts), int(con.shape[0]),
              con.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), por.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
              qor.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    nf = 3 if physics == SHALLOW else (5 if mesh.dim == 3 else 4)
    norms = np.zeros((nf, 6))
    status = ctypes.c_int()
    f = lib().dgmx_restart_diff
    f.argtypes = [ctypes.POINTER(_Mesh), ctypes.c_int, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double,
                  ctypes.c_double, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    st = f(ctypes.byref(m), int(physics), rst1.encode(), rst2.encode(), float(aeps), float(reps), _dp(norms),
           ctypes.byref(status))
    if st != 0:
        raise DgmxError(st, _restart_err())
    return status.value, norms


class _PoolParams(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("flux", ctypes.c_int), ("device", ctypes.c_int),
                ("autotune", ctypes.c_int), ("gamma", ctypes.c_double), ("budget_bytes", ctypes.c_size_t)]


def _pool_lib():
    L = lib()
    if not getattr(L, "_pool_ready", False):
        P, D, I = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int
        L.dgmx_pool_create.argtypes = [ctypes.POINTER(_PoolParams), ctypes.POINTER(P)]
        L.dgmx_pool_destroy.argtypes = [P]
        L.dgmx_pool_prepare.argtypes = [P, I, I, I, I]
        L.dgmx_pool_add.argtypes = [P, ctypes.POINTER(_Mesh), I, D, ctypes.c_double, ctypes.c_double,
                                    ctypes.POINTER(I)]
        L.dgmx_pool_step.argtypes = [P, I]
        L.dgmx_pool_finished.argtypes = [P, ctypes.POINTER(I), I, ctypes.POINTER(I)]
        L.dgmx_pool_get_state.argtypes = [P, I, D]
        L.dgmx_pool_solve_info.argtypes = [P, I, D, ctypes.POINTER(ctypes.c_long), ctypes.POINTER(I)]
        L.dgmx_pool_remove.argtypes = [P, I]
        L.dgmx_pool_stats.argtypes = [P, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(I), ctypes.POINTER(I),
                                      ctypes.POINTER(ctypes.c_longlong)]
        L.dgmx_pool_launch_count.argtypes = [P]
        L.dgmx_pool_launch_count.restype = ctypes.c_long
        L.dgmx_pool_last_error.argtypes = [P]
        L.dgmx_pool_last_error.restype = ctypes.c_char_p
        L._pool_ready = True
    return L


def _mesh_struct(mesh):
    verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
    con = np.ascontiguousarray(mesh.con, dtype=np.int32)
    por = np.ascontiguousarray(mesh.porder, dtype=np.int32)
    qor = np.ascontiguousarray(mesh.qorder, dtype=np.int32)
    m = _Mesh(int(mesh.dim), int(verts.shape[0]), _dp(verts), int(con.shape[0]),
              con.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
              por.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
              qor.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    return m, [verts, con, por, qor]


def _nccl_first():
    # one libnccl.so.2 per process: PyTorch's, loaded before the engine
    # resolves NCCL, so that a later PyTorch import finds the same library
    import torch  # noqa: F401


def nccl_unique_id() -> bytes:
    """A fresh NCCL unique id (rank 0 makes it and shares it with the others)."""
    _nccl_first()
    buf = ctypes.create_string_buffer(128)
    f = lib().dgmx_nccl_unique_id
    f.argtypes = [ctypes.c_char_p]
    st = f(buf)
    if st != 0:
        raise DgmxError(st, lib().dgmx_last_error(None).decode())
    return buf.raw


def partition_plan(mesh, part, nranks: int, rank: int) -> dict:
    """Host-only partition plan of one rank: local and ghost element ids, the
    per-peer block counts and the send / receive block lists."""
    m, keep = _mesh_struct(mesh)
    part = np.ascontiguousarray(part, dtype=np.int32)
    P = ctypes.POINTER(ctypes.c_int)
    f = lib().dgmx_partition_plan
    f.argtypes = [ctypes.c_void_p, P, ctypes.c_int, ctypes.c_int, P, P, P, P, P, P]
    sizes = np.zeros(3, dtype=np.int32)
    ip = lambda a: a.ctypes.data_as(P)
    st = f(ctypes.byref(m), ip(part), int(nranks), int(rank), ip(sizes), None, None, None, None, None)
    if st != 0:
        raise DgmxError(st, lib().dgmx_last_error(None).decode())
    gl, gg = np.zeros(sizes[0], np.int32), np.zeros(sizes[1], np.int32)
    cnt = np.zeros(nranks, np.int32)
    snd, rcv = np.zeros(sizes[2], np.int32), np.zeros(sizes[2], np.int32)
    st = f(ctypes.byref(m), ip(part), int(nranks), int(rank), ip(sizes), ip(gl), ip(gg), ip(cnt), ip(snd), ip(rcv))
    if st != 0:
        raise DgmxError(st, lib().dgmx_last_error(None).decode())
    return {"global_of_local": gl, "global_of_ghost": gg, "peer_counts": cnt, "send": snd, "recv": rcv}


class Group:
    """Every part of an element partition as a handle on one device, stepped
    in lockstep with the halo exchange done by device copies.  State arrays
    are global (Field layout over all elements)."""

    def __init__(self, mesh, physics: int, part, flux: str = "laxfriedrichs", inttype: int = LSRK14,
                 gamma: float = 1.4, vis: float = 0.0, Pr: float = 0.72, device: int = 0, precision: int = FP64,
                 boundaries=None, bulk_hold: bool = False):
        m, self._keep = _mesh_struct(mesh)
        part = np.ascontiguousarray(part, dtype=np.int32)
        self._keep.append(part)
        self.nparts = int(part.max()) + 1
        p = _Params(physics, FLUX[flux.lower()], inttype, precision, 0, device, gamma, vis, Pr)
        L = lib()
        nbc, sides, par = _bc_arrays(boundaries)
        self._keep += [sides, par]
        L.dgmx_group_create_with_boundaries.argtypes = [
            ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int,
            ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
        L.dgmx_group_set_bulk_hold.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.dgmx_group_last_error.restype = ctypes.c_char_p
        L.dgmx_group_last_error.argtypes = [ctypes.c_void_p]
        for n in ("dgmx_group_set_state", "dgmx_group_get_state"):
            getattr(L, n).argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        L.dgmx_group_advance.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.dgmx_group_destroy.argtypes = [ctypes.c_void_p]
        h = ctypes.c_void_p()
        st = L.dgmx_group_create_with_boundaries(
            ctypes.byref(m), ctypes.byref(p), part.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), self.nparts, nbc,
            sides.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), _dp(par), ctypes.byref(h))
        if st != 0:
            raise DgmxError(st, L.dgmx_group_last_error(None).decode())
        self.h = h
        if bulk_hold:
            self._check(L.dgmx_group_set_bulk_hold(self.h, 1))
        self.nf = 3 if physics == SHALLOW else (5 if physics in (EULER3D, NS3D) else 4)
        q = int(mesh.qorder[0]) or int(mesh.porder[0]) + 2
        self.nq = int(mesh.verts.shape[0]) * q ** int(mesh.dim)

    def _check(self, st):
        if st != 0:
            raise DgmxError(st, lib().dgmx_group_last_error(self.h).decode())

    def set_state(self, U):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.nf, self.nq)
        self._check(lib().dgmx_group_set_state(self.h, _dp(U)))

    def state(self):
        U = np.zeros((self.nf, self.nq))
        self._check(lib().dgmx_group_get_state(self.h, _dp(U)))
        return U

    def advance(self, dt: float, nsteps: int = 1):
        self._check(lib().dgmx_group_advance(self.h, float(dt), int(nsteps)))

    def close(self):
        if getattr(self, "h", None):
            lib().dgmx_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PoolFull(DgmxError):
    """The solve does not fit the pool's device-memory budget right now."""


class Pool:
    """Many independent LSRK14 solves on one GPU (include/dgmx_pool.h).

    ``add`` admits a solve (mesh, physics, initial GLL values, step, end
    time); ``step`` advances every unfinished solve; ``finished`` lists the
    solves that reached their end time; ``state`` reads one back.
    """

    def __init__(self, precision: int = FP64, flux: str = "laxfriedrichs", gamma: float = 1.4,
                 budget_bytes: int = 0, autotune: bool = True, device: int = 0, fused: bool = True):
        """fused: the 2-D arenas share one stage launch across orders
        (dgmx_pool_set_fused); False gives every arena its own launches."""
        p = _PoolParams(precision, FLUX[flux.lower()], device, 1 if autotune else 0, gamma, int(budget_bytes))
        h = ctypes.c_void_p()
        st = _pool_lib().dgmx_pool_create(ctypes.byref(p), ctypes.byref(h))
        if st != 0:
            raise DgmxError(st, "pool creation failed")
        self.h = h
        if not fused:
            f = _pool_lib().dgmx_pool_set_fused
            f.argtypes = [ctypes.c_void_p, ctypes.c_int]
            self._check(f(self.h, 0))
        self.nf, self.nq = {}, {}

    def close(self):
        if getattr(self, "h", None):
            _pool_lib().dgmx_pool_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != 0:
            msg = _pool_lib().dgmx_pool_last_error(self.h).decode()
            cls = NonPhysicalState if st == 4 else (PoolFull if st == 6 else DgmxError)
            raise cls(st, msg)

    def prepare(self, physics: int, p: int, q: int = 0, elements: int = 0):
        self._check(_pool_lib().dgmx_pool_prepare(self.h, physics, p, q, elements))

    def add(self, mesh, physics: int, U0, dt: float, t_end: float) -> int:
        verts = np.ascontiguousarray(mesh.verts, dtype=np.float64)
        con = np.ascontiguousarray(mesh.con, dtype=np.int32)
        por = np.ascontiguousarray(mesh.porder, dtype=np.int32)
        qor = np.ascontiguousarray(mesh.qorder, dtype=np.int32)
        ne = int(verts.shape[0])
        nf = 3 if physics == SHALLOW else (5 if mesh.dim == 3 else 4)
        q = int(qor[0]) if qor[0] else int(por[0]) + 2
        nq = ne * q ** mesh.dim
        U0 = np.ascontiguousarray(U0, dtype=np.float64).reshape(nf, nq)
        m = _Mesh(int(mesh.dim), ne, _dp(verts), int(con.shape[0]),
                  con.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                  por.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                  qor.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        sid = ctypes.c_int()
        self._check(_pool_lib().dgmx_pool_add(self.h, ctypes.byref(m), physics, _dp(U0), float(dt),
                                              float(t_end), ctypes.byref(sid)))
        self.nf[sid.value], self.nq[sid.value] = nf, nq
        return sid.value

    def step(self, nsteps: int = 1):
        self._check(_pool_lib().dgmx_pool_step(self.h, int(nsteps)))

    def step_async(self, nsteps: int = 1):
        """Enqueue nsteps steps and return; admission may overlap them.
        Call sync() before finished(), state() or remove()."""
        f = _pool_lib().dgmx_pool_step_async
        f.argtypes = [ctypes.c_void_p, ctypes.c_int]
        self._check(f(self.h, int(nsteps)))

    def sync(self):
        f = _pool_lib().dgmx_pool_sync
        f.argtypes = [ctypes.c_void_p]
        self._check(f(self.h))

    def finished(self):
        buf = (ctypes.c_int * 4096)()
        out, n = [], ctypes.c_int()
        while True:
            self._check(_pool_lib().dgmx_pool_finished(self.h, buf, 4096, ctypes.byref(n)))
            out += list(buf[: n.value])
            if n.value < 4096:
                return out

    def state(self, sid: int):
        U = np.zeros((self.nf[sid], self.nq[sid]))
        self._check(_pool_lib().dgmx_pool_get_state(self.h, int(sid), _dp(U)))
        return U

    def info(self, sid: int):
        """(time, steps taken, finished)."""
        t, s, f = ctypes.c_double(), ctypes.c_long(), ctypes.c_int()
        self._check(_pool_lib().dgmx_pool_solve_info(self.h, int(sid), ctypes.byref(t), ctypes.byref(s),
                                                     ctypes.byref(f)))
        return t.value, s.value, bool(f.value)

    def remove(self, sid: int):
        self._check(_pool_lib().dgmx_pool_remove(self.h, int(sid)))
        self.nf.pop(sid, None)
        self.nq.pop(sid, None)

    def stats(self):
        """(device bytes, resident solves, unfinished solves, unfinished modal DOF)."""
        b, r, a, d = ctypes.c_size_t(), ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        self._check(_pool_lib().dgmx_pool_stats(self.h, ctypes.byref(b), ctypes.byref(r), ctypes.byref(a),
                                                ctypes.byref(d)))
        return b.value, r.value, a.value, d.value

    def launch_count(self) -> int:
        return _pool_lib().dgmx_pool_launch_count(self.h)
