"""dgmx_set_state_async / dgmx_get_state_async: the state calls without the
host wait, as a pipeline of two handles uses them (one solve's transfers
overlapping the other's steps).  Against the synchronous calls on the same
inputs: FP64 bit for bit; the mixed form, whose reference state is then
formed on the device (possibly one rounding apart from the host's), within
1e-9 relative L2."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def pinned(shape):
    import torch
    return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_async_pipeline_equals_sync(precision):
    import dgm_b200
    from oracle import ics
    prec = dgm_b200.MIXED if precision == "mixed" else dgm_b200.FP64
    m = dgm_b200.meshgen.box(3, (6, 6, 6), 0.0, 2 * np.pi, 3)
    A = dgm_b200.Domain(m, dgm_b200.EULER3D, flux="roe", precision=prec)
    B = dgm_b200.Domain(m, dgm_b200.EULER3D, flux="roe", precision=prec)
    ref = dgm_b200.Domain(m, dgm_b200.EULER3D, flux="roe", precision=prec)
    x, y, z = A.coordinates()
    inputs = [ics.taylor_green(x, y, z, Ma=0.1), ics.taylor_green(x, y, z, Ma=0.2)]
    # synchronous chains: each input advanced 2 steps, read back, set again, 2 more
    expect = []
    for U in inputs:
        S = U
        for _ in range(2):
            ref.set_state(S)
            ref.advance(0.002, 2)
            S = ref.state()
        expect.append(S)
    # the same chains through the async calls, the two handles interleaved
    bufs = [pinned(U.shape) for U in inputs]
    for b, U in zip(bufs, inputs):
        b[:] = U
    for _ in range(2):
        for D, b in zip((A, B), bufs):
            D.set_state_async(b)
            D.advance_async(0.002, 2)
            D.state_async(b)
        for D in (A, B):
            D.sync()
    for b, S in zip(bufs, expect):
        if precision == "fp64":
            assert np.array_equal(b, S)
        else:
            assert rel(b, S) < 1e-9
    # pageable memory is refused
    with pytest.raises(dgm_b200.DgmxError):
        A.set_state_async(np.ascontiguousarray(inputs[0]))
    for D in (A, B, ref):
        D.close()
