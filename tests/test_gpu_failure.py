"""Failure detection on the GPU without a fault.

The prefetching stage kernel waits on an mbarrier for each tile's inputs;
every wait is bounded.  These tests make the first wait of every tile run
out (its bound set to zero tries through dgmx_set_wait_limit) and check that
the kernel leaves on its own after letting its copies land, that the call
reports DGMX_ERR_CUDA with the pipeline's message (bit 1 of the device error
word), and that the same context then runs a normal step that matches a
fresh handle bit for bit.  Non-physical states are reported the same way
(bit 0) and leave the context usable too.
"""
import math

import numpy as np
import pytest

from oracle import ics

pytestmark = pytest.mark.gpu


def _pipe_domain(precision):
    import dgm_b200
    mesh = dgm_b200.meshgen.box(3, (4, 4, 4), 0.0, 2 * math.pi, 3)
    D = dgm_b200.Domain(mesh, dgm_b200.EULER3D, flux="roe", inttype=dgm_b200.LSRK14, precision=precision)
    kinds = [D.set_variant(i)[1] for i in range(D.variant_count())]
    assert 2 in kinds, "no prefetching variant compiled for this case"
    pick = kinds.index(2)
    D.set_variant(pick)
    return mesh, D, pick


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_bounded_pipeline_wait_runs_out_and_the_context_recovers(precision):
    import dgm_b200
    mesh, D, pick = _pipe_domain(precision)
    x, y, z = D.coordinates()
    f = ics.taylor_green(x, y, z, Ma=0.1)
    dt = 1e-3
    D.set_state(f)
    D.set_wait_limit(0)
    with pytest.raises(dgm_b200.DgmxError) as ex:
        D.advance(dt, 1)
    assert ex.value.code == 3                     # DGMX_ERR_CUDA
    assert "copy pipeline" in str(ex.value)
    # the same context: restore the bound, start again, step normally
    D.set_wait_limit(-1)
    D.set_state(f)
    D.advance(dt, 2)
    got = D.state()
    R = dgm_b200.Domain(mesh, dgm_b200.EULER3D, flux="roe", inttype=dgm_b200.LSRK14, precision=precision)
    R.set_variant(pick)
    R.set_state(f)
    R.advance(dt, 2)
    assert np.array_equal(got, R.state())
    R.close()
    D.close()


def test_nonphysical_state_is_reported_and_the_context_recovers():
    import dgm_b200
    mesh = dgm_b200.meshgen.box(3, (3, 3, 3), 0.0, 2 * math.pi, 2)
    D = dgm_b200.Domain(mesh, dgm_b200.EULER3D, inttype=dgm_b200.LSRK14)
    x, y, z = D.coordinates()
    f = ics.taylor_green(x, y, z, Ma=0.1)
    bad = f.copy()
    bad[0, : bad.shape[1] // 3] = -1.0            # negative density in the first elements
    D.set_state(bad)
    with pytest.raises(dgm_b200.NonPhysicalState):
        D.advance(1e-3, 1)
    D.set_state(f)
    D.advance(1e-3, 1)
    assert np.isfinite(D.state()).all()
    D.close()
