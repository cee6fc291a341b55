"""The serving loop's latency model (dgm_b200.serving.model_latencies): the
bound the benchmark states comes from it, so its queueing arithmetic is
checked here on cases with known answers (no GPU)."""
import numpy as np

from dgm_b200 import EULER2D
from dgm_b200.requests import Request


def req(arrival, steps, dof_per_step_work):
    # dof such that dof * 14 == the work of one step; dt, t_end give `steps`
    r = Request(EULER2D, 1, 1, t_end=float(steps), arrival=arrival, dt=1.0)
    r.__class__ = type("R", (Request,), {"dof": property(lambda self, w=dof_per_step_work: w / 14)})
    return r


def test_single_request_takes_its_steps_at_capacity():
    from dgm_b200.serving import model_latencies
    lat = model_latencies([req(0.0, 5, 100.0)], capacity=100.0, pass_cost=0.0)
    assert np.allclose(lat, [5.0])


def test_requests_share_passes_and_late_arrivals_wait_for_the_next_pass():
    from dgm_b200.serving import model_latencies
    # two equal requests together: every pass does both steps (2 s), 3 passes
    lat = model_latencies([req(0.0, 3, 100.0), req(0.0, 3, 100.0)], capacity=100.0, pass_cost=0.0)
    assert np.allclose(sorted(lat), [6.0, 6.0])
    # a request arriving during the first pass (0 -> 1 s) joins the second,
    # which carries both (1 -> 3 s)
    lat = model_latencies([req(0.0, 2, 100.0), req(0.5, 1, 100.0)], capacity=100.0, pass_cost=0.0)
    assert np.allclose(sorted(lat), [2.5, 3.0])


def test_pass_cost_adds_per_pass():
    from dgm_b200.serving import model_latencies
    lat = model_latencies([req(0.0, 4, 100.0)], capacity=100.0, pass_cost=0.25)
    assert np.allclose(lat, [5.0])
