"""The allocation-free RHS entry point (dgmx_time_derivative_static).

Callers that cannot allocate device memory on their call path -- a host
callback that may not touch the CUDA API, a real-time loop that forbids
allocation, code whose memory belongs to an arena -- use this entry point:
it keeps the face-trace scratch in a fixed static device array.  This file
runs last so a failure here cannot hide the other tests; it passes alone in
a fresh process and after the rest of the suite.
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
