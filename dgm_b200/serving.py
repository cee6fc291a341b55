"""Batched ensembles and a serving loop over the element pool.

``ensemble_requests`` draws the independent-solve ensemble (Euler 2-D
vortices of random mesh size, order, strength and centre); ``poisson_trace``
draws a request trace with Poisson arrivals mixing shallow-water bumps and
Euler vortices; ``serve`` replays a trace against a ``Pool``: requests are
admitted as they arrive and as device memory allows, every unfinished solve
advances one step per pass (continuous batching: a request that arrives
while others run joins the next pass), finished solves are read back and
released, and each request's latency (arrival to result on the host) is
recorded.  Each pass's step is enqueued first and the arrivals are admitted
while it runs on the GPU.

``calibrate`` and ``model_latencies`` give the latency a request would see
under an ideal schedule of the same kind, from quantities measured apart
from the trace: the pool's throughput on a batch of requests stepped
together, and the fixed cost of one pass.  The model replays the arrivals
through a work-conserving queue in which every admitted request advances one
step per pass and a pass lasts (the steps' work) / throughput + the pass
cost; the stated p99 bound is 1.25 x the model's p99.
"""
from __future__ import annotations

import collections
import math
import time

import numpy as np

from . import EULER2D, SHALLOW, Pool, PoolFull
from .requests import Request, make_request


def ensemble_requests(count: int = 1024, seed: int = 0, n_range=(8, 64), p_range=(2, 7), t_end: float = 1e9,
                      cfl: float = 0.5):
    """Independent 2-D Euler vortex solves: N ~ U{n_range}, p ~ U{p_range},
    beta ~ U[1, 5], centre ~ U[-2, 2]^2 (one generator, seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        p = int(rng.integers(p_range[0], p_range[1] + 1))
        beta = float(rng.uniform(1.0, 5.0))
        x0, y0 = (float(v) for v in rng.uniform(-2.0, 2.0, 2))
        out.append((EULER2D, n, p, t_end, cfl, dict(beta=beta, x0=x0, y0=y0)))
    return out


def poisson_trace(count: int, rate: float = 200.0, seed: int = 0, dof_range=(1e3, 1e6), p_range=(2, 6),
                  t_end_range=(0.5, 5.0), cfl: float = 0.5):
    """Request specs with Poisson(rate) arrivals: half shallow-water bumps
    (a ~ U[0.1, 0.5], w ~ U[0.2, 1], g = 9.81, still water), half Euler
    vortices (beta ~ U[1, 5], centre ~ U[-2, 2]^2); modal DOF log-uniform in
    dof_range (the mesh size N is chosen to match), p ~ U{p_range}, end
    time ~ U[t_end_range]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for _ in range(count):
        t += float(rng.exponential(1.0 / rate))
        sw = bool(rng.random() < 0.5)
        p = int(rng.integers(p_range[0], p_range[1] + 1))
        dof = math.exp(rng.uniform(math.log(dof_range[0]), math.log(dof_range[1])))
        nf = 3 if sw else 4
        n = max(2, int(round(math.sqrt(dof / (nf * (p + 1) ** 2)))))
        t_end = float(rng.uniform(*t_end_range))
        if sw:
            params = dict(a=float(rng.uniform(0.1, 0.5)), w=float(rng.uniform(0.2, 1.0)), g=9.81)
            out.append((SHALLOW, n, p, t_end, cfl, params, t))
        else:
            x0, y0 = (float(v) for v in rng.uniform(-2.0, 2.0, 2))
            params = dict(beta=float(rng.uniform(1.0, 5.0)), x0=x0, y0=y0)
            out.append((EULER2D, n, p, t_end, cfl, params, t))
    return out


def build(spec) -> Request:
    physics, n, p, t_end, cfl, params = spec[:6]
    arrival = spec[6] if len(spec) > 6 else 0.0
    return make_request(physics, n, p, t_end, cfl=cfl, arrival=arrival, **params)


def dof_stages(req: Request, steps: int) -> int:
    """Modal DOF-stage updates of `steps` LSRK14 steps of a request."""
    return req.dof * 14 * steps


def steps_of(req: Request) -> int:
    """Steps a request takes: dt until the last, shortened to land on t_end."""
    return int(math.ceil(req.t_end / req.dt - 1e-12))


def serve(pool: Pool, requests, readback: bool = True, max_wall: float = 600.0):
    """Replays requests (built, sorted by arrival) against the pool in real
    time.  Returns per-request records and the aggregate throughput."""
    pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
    active, records = {}, []
    work = 0
    passes = 0
    t0 = time.perf_counter()

    def admit():
        now = time.perf_counter() - t0
        while pending and pending[0].arrival <= now:
            r = pending[0]
            try:
                sid = pool.add(r.mesh, r.physics, r.U0, r.dt, r.t_end)
            except PoolFull:
                break                      # head of line waits for memory
            pending.popleft()
            active[sid] = (r, time.perf_counter() - t0)

    while pending or active:
        now = time.perf_counter() - t0
        if now > max_wall:
            raise RuntimeError(f"serving did not finish within {max_wall} s")
        if active:
            # the pass's step runs on the GPU while the arrivals are admitted
            pool.step_async(1)
            admit()
            pool.sync()
            passes += 1
            for sid in pool.finished():
                r, admitted = active.pop(sid)
                _, steps, _ = pool.info(sid)
                U = pool.state(sid) if readback else None
                pool.remove(sid)
                done = time.perf_counter() - t0
                work += dof_stages(r, steps)
                records.append(dict(arrival=r.arrival, admitted=admitted, done=done, latency=done - r.arrival,
                                    steps=steps, dof=r.dof, physics=r.physics, p=r.p, n=r.n, state=U))
        else:
            admit()
            if not active and pending:
                time.sleep(max(0.0, min(0.001, pending[0].arrival - (time.perf_counter() - t0))))
    makespan = time.perf_counter() - t0
    lat = np.array([x["latency"] for x in records])
    return dict(records=records, makespan=makespan, dof_stages=work, passes=passes,
                throughput=work / makespan if makespan > 0 else 0.0,
                p50=float(np.percentile(lat, 50)) if lat.size else 0.0,
                p99=float(np.percentile(lat, 99)) if lat.size else 0.0)


def calibrate(pool_factory, requests, batch: int = 48, passes: int = 8):
    """Throughput of the pool on `batch` requests admitted together and
    stepped `passes` times (DOF-stage updates per second, host clock around
    synchronous steps), and the cost of one pass with a single small request
    (launch, synchronisation and bookkeeping).  Measured on pools of their
    own, before and apart from the trace they are used to bound."""
    pool = pool_factory()
    reqs = sorted(requests, key=lambda r: r.arrival)[:batch]
    for r in reqs:
        pool.add(r.mesh, r.physics, r.U0, r.dt, 1e9)
    pool.step(2)
    t0 = time.perf_counter()
    pool.step(passes)
    t = time.perf_counter() - t0
    capacity = sum(r.dof for r in reqs) * 14 * passes / t
    pool.close()
    small = min(requests, key=lambda r: r.dof)
    pool = pool_factory()
    pool.add(small.mesh, small.physics, small.U0, small.dt, 1e9)
    pool.step(3)
    t0 = time.perf_counter()
    pool.step(20)
    pass_cost = (time.perf_counter() - t0) / 20
    pool.close()
    return capacity, pass_cost


def model_latencies(requests, capacity: float, pass_cost: float):
    """Latencies of the requests under the ideal schedule of this kind: a
    request arriving at t joins the first pass that starts after t, advances
    one step per pass, and leaves after its last step; a pass lasts the work
    of the steps it takes / capacity + pass_cost."""
    reqs = sorted(requests, key=lambda r: r.arrival)
    i, t = 0, 0.0
    active = []          # [request, steps left]
    out = []
    while i < len(reqs) or active:
        if not active and i < len(reqs) and reqs[i].arrival > t:
            t = reqs[i].arrival
        while i < len(reqs) and reqs[i].arrival <= t:
            active.append([reqs[i], steps_of(reqs[i])])
            i += 1
        dur = sum(r.dof * 14 for r, _ in active) / capacity + pass_cost
        t += dur
        keep = []
        for item in active:
            item[1] -= 1
            if item[1] <= 0:
                out.append(t - item[0].arrival)
            else:
                keep.append(item)
        active = keep
    return np.array(out)
