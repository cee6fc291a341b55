"""The allocation-free RHS entry point (dgmx_time_derivative_static).

Callers that cannot allocate device memory on their call path -- a
real-time loop that forbids allocation, code whose device memory belongs to
an arena sized once at start-up -- use this entry point from an ordinary
host thread: it keeps the face-trace scratch in a fixed static device array.
This file runs last so a failure here cannot hide the other tests; it passes
alone in a fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _entry():
    import dgm_b200
    L = dgm_b200.lib()
    f = L.dgmx_time_derivative_static
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    g = L.dgmx_time_derivative_device
    g.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    g.restype = ctypes.c_int
    return f, g


@pytest.mark.parametrize("dim,n,p", [(3, (3, 3, 3), 3), (2, (5, 4), 4)])
def test_static_scratch_matches_allocating_entry_point_twice(dim, n, p):
    import torch

    import dgm_b200
    from oracle import ics
    f_static, f_dev = _entry()
    mesh = dgm_b200.meshgen.box(dim, n, 0.0, 2 * np.pi, p)
    phys = dgm_b200.EULER3D if dim == 3 else dgm_b200.EULER2D
    D = dgm_b200.Domain(mesh, phys)
    x, y, z = D.coordinates()
    if dim == 3:
        U = ics.taylor_green(x, y, z, Ma=0.1)
    else:
        U = ics.isentropic_vortex(x - np.pi, y - np.pi, beta=5.0)
    Ud = torch.from_numpy(np.ascontiguousarray(U)).cuda()
    F_ref = torch.zeros_like(Ud)
    assert f_dev(D.h, Ud.data_ptr(), F_ref.data_ptr()) == 0
    D.sync()
    scale = float(F_ref.abs().max()) + float(Ud.abs().max())
    for _ in range(2):  # two calls in a row share the static array
        F = torch.full_like(Ud, float("nan"))
        assert f_static(D.h, Ud.data_ptr(), F.data_ptr()) == 0
        D.sync()
        assert torch.isfinite(F).all()
        assert float((F - F_ref).abs().max()) <= 1e-13 * scale


def test_static_scratch_rejects_meshes_above_its_maximum():
    import torch

    import dgm_b200
    f_static, _ = _entry()
    # 14^3 hexes at p=3: 2744 * 6 faces * 5 fields * 16 points > 2^20 doubles
    mesh = dgm_b200.meshgen.box(3, (14, 14, 14), 0.0, 1.0, 3)
    D = dgm_b200.Domain(mesh, dgm_b200.EULER3D)
    U = torch.ones((5, D.nq), dtype=torch.float64, device="cuda")
    F = torch.zeros_like(U)
    assert f_static(D.h, U.data_ptr(), F.data_ptr()) == 1  # DGMX_ERR_ARGUMENT
    assert b"static scratch maximum" in dgm_b200.lib().dgmx_last_error(D.h)
    assert float(F.abs().max()) == 0.0  # nothing was enqueued


def test_static_scratch_shallow_water_balance_and_source_pulse():
    """Shallow water with the balance capture (the first RHS is stored and
    subtracted from every later one, src/Shallow.cpp:255-266) and a source
    field under a Gaussian time pulse evaluated at Domain::t: each entry
    point on a fresh handle sees the same two calls (capture at U1 and t1,
    then U2 at t2), and the static one repeats the second call."""
    import torch

    import dgm_b200
    from oracle import ics
    f_static, f_dev = _entry()
    mesh = dgm_b200.meshgen.box(2, (6, 5), -2.0, 2.0, 3)
    out = {}
    for name, fn in (("device", f_dev), ("static", f_static)):
        D = dgm_b200.Domain(mesh, dgm_b200.SHALLOW, sw_balance=True)
        x, y, _ = D.coordinates()
        U1 = ics.gaussian_bump(x, y, a=0.3, w=0.6)
        U2 = ics.gaussian_bump(x, y, a=0.25, w=0.5, x0=0.2)
        S = np.zeros_like(U1)
        S[0] = 0.05 * np.exp(-((x - 0.3) ** 2 + (y + 0.1) ** 2) / 0.2)
        D.set_source(S)
        D.set_source_pulse(0.01, 0.004)
        calls = []
        for U, t in ((U1, 0.002), (U2, 0.009), (U2, 0.009)):
            D.set_time(t)
            Ud = torch.from_numpy(np.ascontiguousarray(U)).cuda()
            F = torch.full_like(Ud, float("nan"))
            assert fn(D.h, Ud.data_ptr(), F.data_ptr()) == 0
            D.sync()
            calls.append(F.cpu().numpy())
        out[name] = calls
        D.close()
    ref = out["device"][1]
    scale = float(np.abs(ref).max()) + 1.0
    assert float(np.abs(ref).max()) > 1e-6   # the balance leaves R(U2) - R(U1), not zero
    for F in out["static"][1:]:              # two calls in a row
        assert np.isfinite(F).all()
        assert float(np.abs(F - ref).max()) <= 1e-13 * scale
    assert float(np.abs(out["static"][0] - out["device"][0]).max()) <= 1e-13 * scale


def test_static_scratch_refuses_partitioned_handles():
    import torch

    import dgm_b200
    f_static, _ = _entry()
    mesh = dgm_b200.meshgen.box(3, (2, 2, 2), 0.0, 1.0, 2)
    part = np.arange(8) % 2
    D = dgm_b200.Domain.partition(mesh, dgm_b200.EULER3D, part, 2, 0)
    U = torch.ones((5, D.nq), dtype=torch.float64, device="cuda")
    F = torch.zeros_like(U)
    assert f_static(D.h, U.data_ptr(), F.data_ptr()) == 2  # DGMX_ERR_UNSUPPORTED
    assert b"partitioned" in dgm_b200.lib().dgmx_last_error(D.h)
    D.close()
