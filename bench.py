#!/usr/bin/env python3
"""DOF-stage-updates/s of the B200 DG engine, mixed precision vs FP64 at
matched L2 error, on the 3-D Euler Taylor-Green case; plus the batched
ensemble and the serving loop (p50/p99 latency).

Workload (the single-GPU configuration the metric is quoted on): periodic
[0, 2pi]^3, 32^3 Hex elements, p = 3 (q = 5 GLL points per direction),
compressible Euler, Roe flux, low-storage RK (LSRK14, 14 stages), Mach 0.1
Taylor-Green initial condition.  dt is fixed once from CFL 0.5 on the
initial state.  A "step" is one LSRK14 step (14 fused stage launches).

  value  device-resident throughput of the mixed form (FP32 working
         precision, FP64 solution register): modal DOF x 14 stages x K /
         time (CUDA events on the engine's stream, max over ranks); the
         plain FP64 path is measured the same way under "fp64"
  accuracy  per conserved field, the mixed and FP64 paths against the FP64
         oracle after 10 steps (rank 0, host cores), and the mixed path
         against the GPU FP64 path after the configuration's 500 steps
  e2e    the same metric through the public C ABI with host buffers, for
         both forms: every step uploads the state from pinned host memory
         (dgmx_set_state_async), advances one step (dgmx_advance_async) and
         reads the state back (dgmx_get_state_async), three handles in turn
  roofline  algorithmic bytes per stage launch over its CUDA-event time
         against the measured HBM bandwidth (and, for FP64, algorithmic
         flops against the FP64 FMA rate measured live), with the DRAM
         bytes of one ncu capture from profiles/
  forms  (one GPU) the batched ensemble of 1024 independent 2-D vortex
         solves and a Poisson-arrival serving trace, both through the
         element pool (include/dgmx_pool.h), FP64 and mixed
  other_configs  (rank 0) the 2-D vortex (16^2, p=4) against the oracle,
         the Navier-Stokes Taylor-Green (24^3, p=7, q=9) in FP64, with the
         FP32 viscous kernels and with their 3xTF32 contractions, and the
         reference's channel regression case against its golden restart
Ranks (torchrun, N > 1) run the workload as an element partition, one
z-slab of n^3 elements per GPU on a box that grows with N (weak scaling),
with the face-trace halo after every stage over NCCL, overlapped with the
interior tiles (run_partitioned); --layout replicas runs independent copies
instead, and --transport host stages the halo through the host over gloo.
--impl reference times the CPU restatement of the reference algorithm (the
oracle) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(name="euler3d_taylor_green_32^3_p3_roe_lsrk14", n=32, p=3, q=5, Ma=0.1, gamma=1.4, cfl=0.5,
                flux="roe")
METRIC = "DOF-stage-updates/s mixed vs FP64 at matched L2 err; p50/p99 solve latency"
UNIT = "DOF-stage-updates/s"
# algorithmic bytes per modal DOF and stage: read U, read Ut, write Ut, write U
BYTES_PER_DOF_STAGE = {"fp64": 32, "mixed": 24}   # mixed: U FP64, Ut FP32
# algorithmic flops per modal DOF and stage of the reference algorithm at
# p=3, q=5 (volume gradients, pointwise fluxes, side interpolation and lift,
# one face flux per unique face, projection and update: 81k per element)
FLOPS_PER_DOF_STAGE = 253


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n", type=int, default=WORKLOAD["n"], help="elements per direction")
    ap.add_argument("--no-forms", action="store_true", help="skip the ensemble and serving legs")
    ap.add_argument("--l2-steps", type=int, default=500,
                    help="steps of the mixed-vs-FP64 accuracy run (the configuration's own 500)")
    ap.add_argument("--oracle-steps", type=int, default=10,
                    help="steps of the accuracy run against the FP64 oracle (rank 0, host cores)")
    ap.add_argument("--ensemble", type=int, default=1024, help="solves in the batched ensemble")
    ap.add_argument("--trace", type=int, default=200, help="requests in the serving trace")
    ap.add_argument("--precision", choices=["both", "mixed", "fp64"], default="both",
                    help="time one form only (profiling runs); the default line needs both")
    ap.add_argument("--ns-steps", type=int, default=10,
                    help="steps of the Navier-Stokes Taylor-Green leg (1000 for the full history)")
    ap.add_argument("--only", choices=["vortex2d", "ns3d_tgv", "channel", "ensemble"], default=None,
                    help="run one of the other configurations (or the batched ensemble) alone and print its "
                         "JSON (profiling)")
    ap.add_argument("--variant", type=int, default=-1,
                    help="single-form runs: use this tile variant instead of the autotuner's pick")
    ap.add_argument("--layout", choices=["partition", "replicas"], default="partition",
                    help="N > 1: one element partition per GPU with a halo exchange (weak scaling: the box "
                         "grows by n^3 elements per GPU), or independent replicas")
    ap.add_argument("--transport", choices=["nccl", "host"], default="nccl",
                    help="partitioned halo over NCCL (device buffers, overlapped), or staged through the host "
                         "over a gloo process group (ranks may then share one GPU)")
    return ap.parse_args()


def taylor_green(x, y, z, Ma, gamma):
    p0 = 1.0 / (gamma * Ma * Ma)
    u = np.sin(x) * np.cos(y) * np.cos(z)
    v = -np.cos(x) * np.sin(y) * np.cos(z)
    p = p0 + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0
    E = p / (gamma - 1.0) + 0.5 * (u * u + v * v)
    return np.stack([np.ones_like(x), u, v, np.zeros_like(x), E])


def cfl_dt(U, h, p, gamma, cfl):
    r = U[0]
    u, v, w = U[1] / r, U[2] / r, U[3] / r
    pr = (gamma - 1.0) * (U[4] - 0.5 * r * (u * u + v * v + w * w))
    smax = float(np.max(np.sqrt(u * u + v * v + w * w) + np.sqrt(gamma * pr / r)))
    return cfl * h / ((2 * p + 1) * smax)


def peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(name):
    """DRAM bytes per stage launch from a committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch_full_workload:"):
                return float(line.split(":")[1].split()[0])
    except Exception:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        for l in getattr(self, "lines", []):
            f = [t.strip() for t in l.split(",")]
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except (ValueError, IndexError):
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def build_oracle_problem(n, p, q):
    import oracle
    from oracle import dgm_io
    mesh = dgm_io.box_mesh(3, (n, n, n), 0.0, 2 * math.pi, p, q)
    return oracle.Problem(mesh, oracle.EULER3D, flux=WORKLOAD["flux"])


def cpu_measure(n, p, q, stages_sample, threads):
    """Time the oracle (CPU restatement of the reference algorithm) on a
    bounded sample: `stages_sample` LSRK14 steps of the full workload."""
    import oracle
    oracle.set_threads(threads)
    P = build_oracle_problem(n, p, q)
    x, y, z = P.coords()
    U0 = P.project(taylor_green(x, y, z, WORKLOAD["Ma"], WORKLOAD["gamma"]))
    P.set_state(U0)
    dt = cfl_dt(U0, 2 * math.pi / n, p, WORKLOAD["gamma"], WORKLOAD["cfl"])
    t0 = time.perf_counter()
    P.advance(14, dt, stages_sample)
    t = time.perf_counter() - t0
    dof = 5 * n ** 3 * (p + 1) ** 3
    return dof * 14 * stages_sample / t, t


def config_dict(n, p, q, dof, world=1, layout="partition", transport="nccl"):
    """The workload, identical for both arms (the precision and the tile each
    arm runs are reported outside `config`).  dof: modal DOF per GPU."""
    c = {"workload": WORKLOAD["name"] if n == WORKLOAD["n"] else f"euler3d_taylor_green_{n}^3_p{p}_roe_lsrk14",
         "mesh": f"{n}^3 Hex, periodic [0,2pi]^3", "p": p, "q": q, "physics": "Euler 3-D",
         "flux": "Roe", "integrator": "LSRK14 (14 stages/step)", "Mach": WORKLOAD["Ma"],
         "modal_dof": dof, "cfl": WORKLOAD["cfl"], "parallelism": "single device",
         "l2": "inputs larger than L2 (modal U 84 MB + Ut 42 MB, traces 2x63 MB per GPU in the mixed "
               "form; 168 + 2x126 MB in FP64)"}
    if world > 1 and layout == "partition":
        c["mesh"] = f"{n}x{n}x{n * world} Hex, periodic [0,2pi]^2 x [0,{2 * world}pi]"
        c["modal_dof"] = dof * world
        c["parallelism"] = (f"element partition: {world} z-slabs of {n}^3 elements, one per GPU; halo exchange of "
                            f"the face traces after every stage over "
                            + ("NCCL, overlapped with the interior tiles" if transport == "nccl"
                               else "the host (process group point-to-point)"))
    elif world > 1:
        c["parallelism"] = f"replicas x{world} (independent copies, no halo)"
    return c


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    n, p, q = args.n, WORKLOAD["p"], WORKLOAD["q"]
    threads = os.cpu_count() or 1
    import oracle
    oracle.set_threads(threads)
    P = build_oracle_problem(n, p, q)
    x, y, z = P.coords()
    U0 = P.project(taylor_green(x, y, z, WORKLOAD["Ma"], WORKLOAD["gamma"]))
    P.set_state(U0)
    dt = cfl_dt(U0, 2 * math.pi / n, p, WORKLOAD["gamma"], WORKLOAD["cfl"])
    dof = 5 * n ** 3 * (p + 1) ** 3
    for _ in range(args.warmup):
        P.advance(14, dt, 1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        P.advance(14, dt, 1)
    t = time.perf_counter() - t0
    v = dof * 14 * args.steps / t
    out = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (Taylor-Green initial condition)",
           "config": config_dict(n, p, q, dof, args.gpus, args.layout, args.transport),
           "precision": "FP64 (the oracle: CPU restatement of the reference algorithm)",
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                            "sample": f"{args.steps} LSRK14 steps of the full workload after {args.warmup} warm-up"},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
    return 0


def rel_l2(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def field_errors(S, R):
    """Relative L2 of S against R per conserved field, for the momentum
    vector as one field, of the z-momentum against that vector's norm, and
    over the whole state."""
    return {"per_field": [rel_l2(S[k], R[k]) for k in range(S.shape[0])],
            "momentum_vector": rel_l2(S[1:4], R[1:4]),
            "rho_w_vs_momentum_norm": float(np.linalg.norm(S[3] - R[3]) / max(np.linalg.norm(R[1:4]), 1e-300)),
            "aggregate": rel_l2(S, R)}


def measure_e2e(dgm_b200, D, stream, prec, mesh, local, variant, dt, args, barrier, max_over_ranks, world, dof):
    """The metric through the public C ABI with host buffers: per step the
    state is uploaded from pinned host memory (and projected), advanced one
    LSRK14 step and read back.  Serial on one handle, and as a pipeline of
    three handles (the asynchronous state calls) so one solve's upload and
    another's read-back overlap the third's step on separate copy engines."""
    import torch
    Uh = torch.empty((5, D.nq), dtype=torch.float64, pin_memory=True).numpy()
    Uh[:] = D.state()
    for _ in range(max(1, args.warmup)):
        D.set_state(Uh)
        D.advance(dt, 1)
        D.state_into(Uh)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ke = max(3, args.steps // 2)
    e0.record(stream)
    for _ in range(ke):
        D.set_state(Uh)
        D.advance(dt, 1)
        D.state_into(Uh)
    e1.record(stream)
    e1.synchronize()
    barrier()
    te = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    e2e_serial = world * dof * 14 * ke / te
    nbytes = 5 * D.nq * 8
    extra = [dgm_b200.Domain(mesh, dgm_b200.EULER3D, flux=WORKLOAD["flux"], inttype=dgm_b200.LSRK14,
                             device=local, precision=prec) for _ in range(2)]
    for X in extra:
        X.set_variant(variant)
    pair = (D, *extra)
    xs = [torch.cuda.ExternalStream(X.stream(), device=torch.device("cuda", local)) for X in extra]
    bufs = [torch.empty((5, D.nq), dtype=torch.float64, pin_memory=True).numpy() for _ in pair]
    for b in bufs:
        b[:] = Uh

    def pipeline(k):
        for i in range(k):
            X, b = pair[i % len(pair)], bufs[i % len(pair)]
            X.sync()                       # its previous read-back has landed in b
            X.set_state_async(b)
            X.advance_async(dt, 1)
            X.state_async(b)

    pipeline(len(pair) * max(1, args.warmup))
    for X in pair:
        X.sync()
    barrier()
    kp = 3 * ke
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for sx in xs:
        sx.wait_event(e0)
    pipeline(kp)
    for sx in xs:
        ex = torch.cuda.Event()
        ex.record(sx)
        stream.wait_event(ex)
    e1.record(stream)
    e1.synchronize()
    for X in pair:
        X.sync()
    barrier()
    tp = max_over_ranks(e0.elapsed_time(e1) / 1e3)
    for X in extra:
        X.close()
    return {"value": world * dof * 14 * kp / tp, "unit": UNIT, "h2d_bytes_per_step": nbytes,
            "d2h_bytes_per_step": nbytes, "steps": kp,
            "path": "per step: dgmx_set_state_async (pinned host -> device, projection) + dgmx_advance_async "
                    "(1 step) + dgmx_get_state_async (device -> pinned host), three handles in turn so uploads "
                    "and read-backs overlap steps; device time from the first upload to the last read-back",
            "serial": {"value": e2e_serial, "steps": ke,
                       "path": "dgmx_set_state + dgmx_advance(1 step) + dgmx_get_state on one handle"}}


def time_steps(D, stream, dt, steps, warmup, barrier, max_over_ranks, clk=None):
    """Device time of `steps` LSRK14 steps (CUDA events on the engine's stream)."""
    import torch
    for _ in range(warmup):
        D.advance_async(dt, 1)
    D.sync()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = D.launch_count()
    if clk is not None:
        clk.__enter__()
    ev0.record(stream)
    for _ in range(steps):
        D.advance_async(dt, 1)
    ev1.record(stream)
    ev1.synchronize()
    if clk is not None:
        clk.__exit__(None, None, None)
    launches = D.launch_count() - l0
    D.sync()
    barrier()
    return max_over_ranks(ev0.elapsed_time(ev1) / 1e3), launches


def other_configs(dgm_b200, args, only=None):
    """The other benchmark cases on this GPU.  The 2-D isentropic
    vortex (16 x 16 Quads on [-5,5]^2, p=4, beta=5, LF, LSRK14, dt from CFL
    0.5, 200 steps) with its L2 distance from the FP64 oracle and from the
    exact (advected) vortex per conserved field, at q=6 (the reference's
    default q=p+2) and q=5; at q=5 the under-integrated scheme loses
    positivity in the oracle as well, so that leg reports the step block in
    which each run first reports a non-physical state.  The 3-D
    Navier-Stokes Taylor-Green vortex (24^3 Hex, p=7, q=9, Re=1600, Pr=0.71,
    Mach 0.1, Roe, LSRK14) timed over its first steps, with the
    kinetic-energy history (FP64).  And the reference's runs/chan regression
    case (walls, bulk-flow hold) against its golden restart.  `only` runs one
    of them."""
    import torch
    from dgm_b200 import requests as R
    res = {}
    if only in (None, "vortex2d"):
        n, p, steps, block = 16, 4, 200, 10
        for q in (6, 5):
            mesh = dgm_b200.meshgen.box(2, (n, n), -5.0, 5.0, p, q)
            D = dgm_b200.Domain(mesh, dgm_b200.EULER2D, flux="laxfriedrichs", inttype=dgm_b200.LSRK14)
            x, y = D.coordinates()[:2]
            U0 = R.vortex(x, y, beta=5.0)
            dt = R.cfl_dt(U0, 10.0 / n, p, dgm_b200.EULER2D, 0.5)
            c1 = {"workload": f"euler2d_isentropic_vortex_16^2_p4_q{q}_lf_lsrk14_{steps}steps", "dt": dt}
            D.set_state(U0)
            gpu_fail = None
            if q == 6:
                D.advance(dt, 3)
                D.set_state(U0)
                st = torch.cuda.ExternalStream(D.stream())
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                D.advance_async(dt, steps)
                e1.record(st)
                e1.synchronize()
                D.sync()
                t = e0.elapsed_time(e1) / 1e3
                c1.update({"value": 4 * n * n * (p + 1) ** 2 * 14 * steps / t, "unit": UNIT,
                           "ms_per_step": 1e3 * t / steps})
            else:
                for b in range(steps // block):
                    try:
                        D.advance(dt, block)
                    except dgm_b200.NonPhysicalState:
                        gpu_fail = (b + 1) * block
                        break
            if not args.no_cpu_baseline:
                import oracle
                from oracle import dgm_io
                P = oracle.Problem(dgm_io.Mesh(2, mesh.verts, mesh.con, mesh.porder, mesh.qorder), oracle.EULER2D)
                P.set_state(P.project(U0))
                if q == 6:
                    P.advance(14, dt, steps)
                    G, O = D.state(), P.state()
                    c1["rel_l2_vs_oracle_per_field"] = [rel_l2(G[k], O[k]) for k in range(4)]
                else:
                    ora_fail = None
                    for b in range(steps // block):
                        if P.advance(14, dt, block) != 0:
                            ora_fail = (b + 1) * block
                            break
                    c1["nonphysical_within_steps"] = {"gpu": gpu_fail, "oracle": ora_fail}
            if q == 6:
                # the vortex rides the free stream (u=1, v=0): the exact state at T is the initial one shifted by T
                c1["rel_l2_vs_exact_per_field"] = [rel_l2(a, b) for a, b in
                                                   zip(D.state(), R.vortex(x, y, beta=5.0, x0=dt * steps))]
            D.close()
            res[f"vortex2d_q{q}"] = c1
    if only in (None, "ns3d_tgv"):
        # Navier-Stokes Taylor-Green, 24^3, p=7, q=p+2 (the reference's
        # default quadrature; at q=p+1 grid-scale noise grows without bound)
        n, p, q, k3 = 24, 7, 9, max(1, args.ns_steps)
        stride = max(1, k3 // 100)   # kinetic-energy samples: at most ~100 besides t=0
        mesh = dgm_b200.meshgen.box(3, (n, n, n), 0.0, 2 * math.pi, p, q)
        D = dgm_b200.Domain(mesh, dgm_b200.NS3D, flux="roe", inttype=dgm_b200.LSRK14, vis=1.0 / 1600.0, Pr=0.71)
        x, y, z = D.coordinates()
        U0 = taylor_green(x, y, z, 0.1, 1.4)
        dt = cfl_dt(U0, 2 * math.pi / n, p, 1.4, 0.5)
        D.set_state(U0)
        rows, _ = D.autotune(reps=3)
        D.set_state(U0)
        xg = R.gll_points(q)
        c = np.zeros(q)
        c[-1] = 1.0
        w1 = 2.0 / ((q - 1) * q * np.polynomial.legendre.legval(xg, c) ** 2)
        w = np.einsum("i,j,k->kji", w1, w1, w1).reshape(-1)

        def kinetic_energy(U):
            # volume mean of rho |u|^2 / 2 (GLL quadrature; equal elements)
            e = 0.5 * (U[1] ** 2 + U[2] ** 2 + U[3] ** 2) / U[0]
            return float((e.reshape(-1, q ** 3) * w).sum() / (w.sum() * e.size / q ** 3))

        def timed_steps(D):
            st = torch.cuda.ExternalStream(D.stream())
            ke, t = [kinetic_energy(D.state())], 0.0
            for i in range(k3):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(st)
                D.advance_async(dt, 1)
                e1.record(st)
                e1.synchronize()
                D.sync()
                t += e0.elapsed_time(e1) / 1e3
                if (i + 1) % stride == 0 or i + 1 == k3:
                    ke.append(kinetic_energy(D.state()))
            return t, ke

        t, ke = timed_steps(D)
        dof = 5 * n ** 3 * (p + 1) ** 3
        res["ns3d_tgv"] = {"workload": "ns3d_taylor_green_24^3_p7_q9_re1600_pr0.71_roe_lsrk14", "steps_timed": k3,
                          "dt": dt, "value": dof * 14 * k3 / t, "unit": UNIT, "ms_per_step": 1e3 * t / k3,
                          "kinetic_energy": ke, "kinetic_energy_every_steps": stride,
                          "tile_us": [round(float(r[3]), 1) for r in rows],
                          # -dKE/dt at t=0 of the incompressible limit is nu <|grad u|^2> = 3 nu / 4
                          "dissipation_rate": (ke[0] - ke[-1]) / (k3 * dt), "dissipation_rate_t0_exact": 0.75 / 1600.0,
                          "note": "FP64 BR1" + ("" if k3 >= 1000 else "; --ns-steps 1000 runs the full history")}
        U64 = D.state()
        D.close()
        # the FP32 viscous form (precision MIXED): BR1 gradient and viscous
        # kernels in FP32, stage kernel, registers and traces in FP64
        D = dgm_b200.Domain(mesh, dgm_b200.NS3D, flux="roe", inttype=dgm_b200.LSRK14, vis=1.0 / 1600.0, Pr=0.71,
                            precision=dgm_b200.MIXED)
        D.set_state(U0)
        D.advance(dt, 3)
        D.set_state(U0)
        t32, ke32 = timed_steps(D)
        res["ns3d_tgv_fp32_viscous"] = {
            "workload": "ns3d_taylor_green_24^3_p7_q9_re1600_pr0.71_roe_lsrk14", "steps_timed": k3,
            "value": dof * 14 * k3 / t32, "unit": UNIT, "ms_per_step": 1e3 * t32 / k3,
            "rel_l2_vs_fp64_per_field": [rel_l2(a, b) for a, b in zip(D.state(), U64)],
            "kinetic_energy_rel_diff_vs_fp64": abs(ke32[-1] - ke[-1]) / ke[-1],
            "kinetic_energy_max_rel_diff_vs_fp64": max(abs(a - b) / b for a, b in zip(ke32, ke))}
        # the same with the viscous kernels' 1-D contractions as 3xTF32
        # tensor-core products
        D.set_tensor_contractions(True)
        D.set_state(U0)
        D.advance(dt, 3)
        D.set_state(U0)
        ttc, ketc = timed_steps(D)
        res["ns3d_tgv_3xtf32_viscous"] = {
            "workload": "ns3d_taylor_green_24^3_p7_q9_re1600_pr0.71_roe_lsrk14", "steps_timed": k3,
            "value": dof * 14 * k3 / ttc, "unit": UNIT, "ms_per_step": 1e3 * ttc / k3,
            "rel_l2_vs_fp64_per_field": [rel_l2(a, b) for a, b in zip(D.state(), U64)],
            "kinetic_energy_rel_diff_vs_fp64": abs(ketc[-1] - ke[-1]) / ke[-1],
            "note": "FP32 viscous kernels with their contractions on the tensor cores (mma.sync m16n8k8 TF32, "
                    "3 products per contraction: small x big + big x small + big x big)"}
        D.close()
    if only in (None, "channel"):
        # the reference's channel regression case (runs/chan: NS 3-D, 512 hexes, p=3,
        # isothermal walls, bulk-flow hold, TVD3, 100 steps from its restart initial
        # condition), inputs and golden result from the committed fixture
        z = np.load(os.path.join(ROOT, "tests", "golden", "chan.npz"))
        meta = json.loads(str(z["meta"]))
        inp = meta["inp"]
        mesh = dgm_b200.meshgen.Mesh(3, z["verts"], z["con"], z["porder"], z["qorder"])
        tw, eref = meta["bct"][meta["bc_tags"][0]][1][:2]
        rec = [(int(e), int(s_), dgm_b200.BC_ISOTHERMAL_WALL, tw, eref) for e, s_ in z["bc_sides"]]
        D = dgm_b200.Domain(mesh, dgm_b200.NS3D, inttype=inp["inttype"], vis=float(inp["vis"]), boundaries=rec,
                            bulk_hold=True)
        D.set_modes(z["ic_modal"])
        D.advance(float(inp["dt"]), 2)
        D.set_modes(z["ic_modal"])
        st = torch.cuda.ExternalStream(D.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        D.advance_async(float(inp["dt"]), int(inp["Nt"]))
        e1.record(st)
        e1.synchronize()
        D.sync()
        t = e0.elapsed_time(e1) / 1e3
        nsteps = int(inp["Nt"])
        dof = 5 * mesh.verts.shape[0] * 64
        chan = {"workload": "runs/chan (NS 3-D channel, 512 hexes, p=3, isothermal walls, bulk-flow hold, TVD3)",
                "steps": nsteps, "ms_per_step": 1e3 * t / nsteps, "value": dof * 3 * nsteps / t, "unit": UNIT,
                "max_abs_modal_diff_vs_golden": float(np.abs(D.modes() - z["modal"]).max())}
        D.close()
        if not args.no_cpu_baseline:
            import oracle
            from oracle import dgm_io
            oracle.set_threads(os.cpu_count() or 1)
            P = oracle.Problem(dgm_io.Mesh(3, mesh.verts, mesh.con, mesh.porder, mesh.qorder), oracle.NS3D,
                               vis=float(inp["vis"]))
            P.set_bc(rec)
            P.set_hold_bulk(True)
            P.set_state(P.backward(z["ic_modal"]))
            t0 = time.perf_counter()
            P.advance(3, float(inp["dt"]), nsteps)
            tc = time.perf_counter() - t0
            chan["cpu_oracle_ms_per_step"] = 1e3 * tc / nsteps
            chan["cpu_oracle_cores"] = os.cpu_count() or 1
        res["channel"] = chan
    return res


def forms(dgm_b200, args, serve=True):
    """The batched ensemble and (serve) the serving trace on this GPU (pool
    path)."""
    from dgm_b200 import serving
    res = {}
    specs = serving.ensemble_requests(args.ensemble, seed=0)
    ens = {}
    for name, prec in (("fp64", dgm_b200.FP64), ("mixed", dgm_b200.MIXED)):
        for path in ("fused", "per_arena"):
            pool = dgm_b200.Pool(prec, fused=path == "fused")
            dof = 0
            t0 = time.perf_counter()
            for spec in specs:
                r = serving.build(spec)
                pool.add(r.mesh, r.physics, r.U0, r.dt, r.t_end)
                dof += r.dof
            setup = time.perf_counter() - t0
            pool.step(3)
            l0 = pool.launch_count()
            k = 5
            t0 = time.perf_counter()
            pool.step(k)            # returns after the GPU has finished
            t = time.perf_counter() - t0
            row = {"value": dof * 14 * k / t, "unit": UNIT, "ms_per_step": 1e3 * t / k,
                   "device_bytes": pool.stats()[0], "launches_per_step": (pool.launch_count() - l0) // k,
                   "admission_s": round(setup, 2)}
            pool.close()
            if path == "fused":
                ens[name] = row
            else:
                ens[name]["per_arena"] = row
    ens["speedup_mixed_vs_fp64"] = ens["mixed"]["value"] / ens["fp64"]["value"]
    ens["config"] = {"solves": args.ensemble, "modal_dof": dof, "physics": "Euler 2-D isentropic vortex, LF",
                     "mesh": "N x N periodic Quad on [-5,5]^2, N ~ U{8..64}", "p": "U{2..7}, q = p+2",
                     "beta": "U[1,5]", "centre": "U[-2,2]^2", "seed": 0,
                     "launch": "one persistent launch per LSRK stage for every order together (the fused "
                               "multi-order stage kernel over (arena, tile) work items), one CUDA graph per step; "
                               "'per_arena': one persistent launch per (order) arena per stage, arenas on concurrent "
                               "streams, tiles autotuned per (physics, p)",
                     "timing": f"{k} steps after 3, host clock around synchronous pool steps"}
    res["ensemble"] = ens
    if not serve:
        return res

    trace = serving.poisson_trace(args.trace, rate=200.0, seed=1)
    reqs = [serving.build(s) for s in trace]
    work = sum(r.dof * 14 * serving.steps_of(r) for r in reqs)
    span = reqs[-1].arrival
    srv = {}
    for name, prec in (("mixed", dgm_b200.MIXED), ("fp64", dgm_b200.FP64)):
        def factory(prec=prec):
            pool = dgm_b200.Pool(prec, budget_bytes=40 << 30)
            for ph in (dgm_b200.EULER2D, dgm_b200.SHALLOW):
                for p in range(2, 7):
                    pool.prepare(ph, p, 0, 4096)
            return pool
        # the bound: a work-conserving model of the same schedule with the
        # pool's throughput and pass cost measured apart from the trace
        capacity, pass_cost = serving.calibrate(factory, reqs, batch=64)
        model = serving.model_latencies(reqs, capacity, pass_cost)
        bound = 1.25 * float(np.percentile(model, 99))
        pool = factory()
        out = serving.serve(pool, reqs, readback=True)
        # alone vs in the mix: re-run three served requests alone, compare
        same = True
        for rec_i in (0, len(out["records"]) // 2, len(out["records"]) - 1):
            rec = sorted(out["records"], key=lambda x: x["arrival"])[rec_i]
            r = next(q for q in reqs if q.arrival == rec["arrival"])
            solo = dgm_b200.Pool(prec)
            sid = solo.add(r.mesh, r.physics, r.U0, r.dt, r.t_end)
            while not solo.info(sid)[2]:
                solo.step(50)
            same = same and bool(np.array_equal(solo.state(sid), rec["state"]))
            solo.close()
        lat = np.array([x["latency"] for x in out["records"]])
        srv[name] = {"p50_s": out["p50"], "p99_s": out["p99"], "p90_s": float(np.percentile(lat, 90)),
                     "max_s": float(lat.max()), "throughput": out["throughput"], "unit": UNIT,
                     "makespan_s": out["makespan"], "passes": out["passes"], "p99_bound_s": bound,
                     "model": {"p50_s": float(np.percentile(model, 50)), "p99_s": float(np.percentile(model, 99)),
                               "capacity": capacity, "pass_cost_s": pass_cost},
                     "meets_p99_bound": bool(out["p99"] <= bound), "alone_equals_mix": same}
        pool.close()
    srv["config"] = {"requests": len(reqs), "rate_per_s": 200.0, "arrival_span_s": span, "seed": 1,
                     "mix": "1/2 shallow-water Gaussian bump (a~U[0.1,0.5], w~U[0.2,1], g=9.81, still water), "
                            "1/2 Euler vortex (beta~U[1,5], centre~U[-2,2]^2)",
                     "dof": "log-uniform 1e3..1e6 modal", "p": "U{2..6}", "t_end": "U[0.5,5]",
                     "budget_bytes": 40 << 30, "offered_work_dof_stages": work,
                     "p99_bound": "1.25 x the p99 of a work-conserving model of the same schedule (every admitted "
                                  "request advances one step per pass; a pass lasts its steps' work / capacity + the "
                                  "pass cost), with the capacity (64 requests of the trace stepped together) and the "
                                  "pass cost (one small request) measured on separate pools before the trace",
                     "loop": "each pass enqueues its step (dgmx_pool_step_async) and admits the arrivals while it "
                             "runs, then syncs, reads back and releases the finished requests",
                     "latency": "arrival to state read back on the host, wall clock"}
    res["serving"] = srv
    return res


def run_partitioned(args, torch, dgm_b200, dist, rank, world, local):
    """N > 1: the workload as an element partition, one rank per GPU (weak
    scaling).  The Taylor-Green box grows along z to n x n x nN elements over
    [0,2pi]^2 x [0,2pi N] (the initial condition is 2pi-periodic, so every
    rank's slab of n^3 elements holds the single-GPU problem), rank r owns the
    z-slab r, and after every stage the face traces on the slab faces cross to
    the neighbouring ranks: over NCCL from device buffers while the interior
    tiles run (dgmx_set_exchange_nccl, the overlapped stage), or with
    --transport host through pinned host memory and the process group.  Both
    forms (FP64 and mixed) are timed on the device (CUDA events on the
    engine's stream, max over ranks); e2e uploads every rank's state from
    pinned host memory, advances one step and reads it back.  The partitioned
    state equals the unpartitioned one bit for bit (tests/test_gpu_partition.py),
    so the accuracy figures are those of the single-GPU line."""
    n, p, q = args.n, WORKLOAD["p"], WORKLOAD["q"]
    host = args.transport == "host"
    L = 2 * math.pi
    mesh = dgm_b200.meshgen.box(3, (n, n, n * world), 0.0, (L, L, L * world), p, q)
    part = (np.arange(n ** 3 * world) // n ** 3).astype(np.int32)   # element e = i + n (j + n k): z-slabs
    dof = 5 * n ** 3 * (p + 1) ** 3                                  # per rank

    def barrier():
        dist.barrier()
        torch.cuda.synchronize()

    def reduce(v, op):
        t = torch.tensor([v], dtype=torch.float64, device="cpu" if host else "cuda")
        dist.all_reduce(t, op=op)
        return float(t.item())

    def max_over_ranks(v):
        return reduce(v, dist.ReduceOp.MAX)

    doms, tiles = {}, {}
    U_ic = dt = None
    for name, prec in (("fp64", dgm_b200.FP64), ("mixed", dgm_b200.MIXED)):
        D = dgm_b200.Domain.partition(mesh, dgm_b200.EULER3D, part, world, rank, flux=WORKLOAD["flux"],
                                      inttype=dgm_b200.LSRK14, device=local, precision=prec)
        if host:
            D.set_exchange_host()
        else:   # one NCCL communicator per handle, each from its own id
            obj = [dgm_b200.nccl_unique_id() if rank == 0 else None]
            dist.broadcast_object_list(obj, src=0)
            D.set_exchange_nccl(obj[0])
        if U_ic is None:
            x, y, z = D.coordinates()
            U_ic = taylor_green(x, y, z, WORKLOAD["Ma"], WORKLOAD["gamma"])
            dt = -reduce(-cfl_dt(U_ic, L / n, p, WORKLOAD["gamma"], WORKLOAD["cfl"]), dist.ReduceOp.MAX)
        D.set_state(U_ic)
        rows, pick = D.autotune(reps=10)
        pick = int(-reduce(-pick, dist.ReduceOp.MAX))   # one tile for every rank (rank-order independent)
        _, kind = D.set_variant(pick)
        D.set_state(U_ic)
        tiles[name] = {"variant": pick,
                       "kernel": {2: "stage_pipe_kernel", 3: "stage2_kernel"}.get(kind, "stage_kernel"),
                       "elements_per_cta": int(rows[pick][0]), "min_ctas_per_sm": int(rows[pick][1]),
                       "threads_per_cta": int(rows[pick][2])}
        doms[name] = D
    streams = {k: torch.cuda.ExternalStream(D.stream(), device=torch.device("cuda", local)) for k, D in doms.items()}
    clk = ClockSampler(local)
    t64, _ = time_steps(doms["fp64"], streams["fp64"], dt, args.steps, args.warmup, barrier, max_over_ranks)
    tmx, launches = time_steps(doms["mixed"], streams["mixed"], dt, args.steps, args.warmup, barrier,
                               max_over_ranks, clk)
    value = world * dof * 14 * args.steps / tmx
    v64 = world * dof * 14 * args.steps / t64

    def e2e(D, stream):
        Uh = torch.empty((5, D.nq), dtype=torch.float64, pin_memory=True).numpy()
        Uh[:] = U_ic
        for _ in range(max(1, args.warmup)):
            D.set_state(Uh)
            D.advance(dt, 1)
            D.state_into(Uh)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k = max(3, args.steps // 2)
        e0.record(stream)
        for _ in range(k):
            D.set_state(Uh)
            D.advance(dt, 1)
            D.state_into(Uh)
        e1.record(stream)
        e1.synchronize()
        barrier()
        t = max_over_ranks(e0.elapsed_time(e1) / 1e3)
        nbytes = world * 5 * D.nq * 8
        return {"value": world * dof * 14 * k / t, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes, "steps": k,
                "path": "per step on every rank: dgmx_set_state (pinned host -> device, projection, reference "
                        "state and traces with their halo) + dgmx_advance (1 step) + dgmx_get_state (device -> "
                        "pinned host); bytes summed over the ranks"}

    e2e_res = {name: e2e(D, streams[name]) for name, D in doms.items()}
    peak, pkind = peaks()
    stage_mx, stage_64 = tmx / (14 * args.steps), t64 / (14 * args.steps)

    def roof(prec, stage_s, prof):
        a = BYTES_PER_DOF_STAGE[prec] * dof / stage_s / 1e9
        return {"bound": "hbm", "achieved": a, "peak": peak, "unit": "GB/s", "frac": a / peak,
                "peak_kind": pkind, "traffic": profile_traffic(prof),
                "kernel": f"{tiles[prec]['kernel']}<Euler3D, L=4, Q=5, {prec}> (boundary and interior tiles of "
                          f"one rank, per GPU; the stage time includes the halo)",
                "algorithmic_bytes_per_launch": BYTES_PER_DOF_STAGE[prec] * dof, "stage_us": 1e6 * stage_s}

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tmx / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 solution register)",
           "data": "synthetic (Taylor-Green initial condition, no dataset)",
           "config": config_dict(n, p, q, dof, world, "partition", args.transport),
           "precision": "mixed: FP32 states, fluxes and contractions, FP64 solution register",
           "tile": tiles["mixed"],
           "fp64": {"value": v64, "unit": UNIT, "ms_per_step": 1e3 * t64 / args.steps, "tile": tiles["fp64"],
                    "roofline": roof("fp64", stage_64, "euler3d_tgv_p3_stage_kernel.md"), "e2e": e2e_res["fp64"]},
           "speedup_mixed_vs_fp64": value / v64,
           "accuracy": {"note": "the partitioned state equals the unpartitioned one bit for bit in both forms "
                                "(tests/test_gpu_partition.py); the per-field errors are the single-GPU line's"},
           "e2e": e2e_res["mixed"],
           "gpu_launches": int(launches), "clocks": clk.summary(),
           "roofline": roof("mixed", stage_mx, "euler3d_tgv_p3_stage_mixed.md")}
    for D in doms.values():
        D.close()
    if rank == 0:
        print(json.dumps(out), flush=True)
    dist.barrier()
    dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import dgm_b200
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.layout == "partition" and args.transport == "host":
        local %= max(1, torch.cuda.device_count())   # host-staged ranks may share a GPU (no kernel waits on a peer)
    torch.cuda.set_device(local)
    if args.only:
        if rank == 0:
            res = forms(dgm_b200, args, serve=False) if args.only == "ensemble" else \
                other_configs(dgm_b200, args, args.only)
            print(json.dumps(res), flush=True)
        return 0
    dist = None
    host_pg = world > 1 and args.layout == "partition" and args.transport == "host"
    if world > 1:
        import datetime
        import torch.distributed as dist
        if host_pg:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
        else:
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
    if world > 1 and args.layout == "partition":
        return run_partitioned(args, torch, dgm_b200, dist, rank, world, local)
    n, p, q = args.n, WORKLOAD["p"], WORKLOAD["q"]
    mesh = dgm_b200.meshgen.box(3, (n, n, n), 0.0, 2 * math.pi, p, q)
    dof = 5 * n ** 3 * (p + 1) ** 3

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    doms, tiles, results = {}, {}, {}
    U_ic = dt = None
    forms_run = [(k, v) for k, v in (("fp64", dgm_b200.FP64), ("mixed", dgm_b200.MIXED))
                 if args.precision in ("both", k)]
    for name, prec in forms_run:
        D = dgm_b200.Domain(mesh, dgm_b200.EULER3D, flux=WORKLOAD["flux"], inttype=dgm_b200.LSRK14,
                            device=local, precision=prec)
        if U_ic is None:
            x, y, z = D.coordinates()
            U_ic = taylor_green(x, y, z, WORKLOAD["Ma"], WORKLOAD["gamma"])
            dt = cfl_dt(U_ic, 2 * math.pi / n, p, WORKLOAD["gamma"], WORKLOAD["cfl"])
        D.set_state(U_ic)
        # tile autotuning is set-up, outside the timed region
        rows, pick = D.autotune(reps=10)
        if args.precision != "both" and args.variant >= 0:
            pick = args.variant
        _, kind = D.set_variant(pick)
        tiles[name] = {"variant": pick,
                       "kernel": {2: "stage_pipe_kernel", 3: "stage2_kernel"}.get(kind, "stage_kernel"),
                       "elements_per_cta": int(rows[pick][0]), "min_ctas_per_sm": int(rows[pick][1]),
                       "threads_per_cta": int(rows[pick][2]), "candidates_us": [round(float(r[3]), 1) for r in rows]}
        doms[name] = D
    streams = {k: torch.cuda.ExternalStream(D.stream(), device=torch.device("cuda", local)) for k, D in doms.items()}

    clk = ClockSampler(local)
    if args.precision != "both":
        # one form alone (profiling): its device time, nothing else
        t1, _ = time_steps(doms[args.precision], streams[args.precision], dt, args.steps, args.warmup, barrier,
                           max_over_ranks)
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": world * dof * 14 * args.steps / t1, "unit": UNIT,
                              "precision": args.precision, "ms_per_step": 1e3 * t1 / args.steps,
                              "tile": tiles[args.precision], "note": "single-form profiling run"}), flush=True)
        for Dx in doms.values():
            Dx.close()
        if dist is not None:
            dist.destroy_process_group()
        return 0
    t64, _ = time_steps(doms["fp64"], streams["fp64"], dt, args.steps, args.warmup, barrier, max_over_ranks)
    tmx, launches = time_steps(doms["mixed"], streams["mixed"], dt, args.steps, args.warmup, barrier,
                               max_over_ranks, clk)
    value = world * dof * 14 * args.steps / tmx
    v64 = world * dof * 14 * args.steps / t64

    # accuracy: mixed and FP64 against the FP64 oracle over the first steps
    # (one rank), and mixed against the FP64 path (itself within 1e-12 of the
    # oracle, tests/test_gpu_parity_at_size.py) over the configuration's own
    # step count
    accuracy = {}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.oracle_steps > 0:
        import oracle
        oracle.set_threads(os.cpu_count() or 1)
        P = build_oracle_problem(n, p, q)
        P.set_state(P.project(U_ic))
        t0 = time.perf_counter()
        P.advance(14, dt, args.oracle_steps)
        O = P.state()
        to = time.perf_counter() - t0
        row = {"steps": args.oracle_steps, "t": args.oracle_steps * dt, "oracle_s": round(to, 1)}
        for name, D in doms.items():
            D.set_state(U_ic)
            D.advance(dt, args.oracle_steps)
            row[name] = field_errors(D.state(), O)
        del P
        accuracy["vs_fp64_oracle"] = row
    for D in doms.values():
        D.set_state(U_ic)
        D.advance(dt, args.l2_steps)
    S64, Smx = doms["fp64"].state(), doms["mixed"].state()
    accuracy["mixed_vs_fp64"] = {"steps": args.l2_steps, "t": args.l2_steps * dt, **field_errors(Smx, S64),
                                 "rel_l2_of_state_change_fp64": rel_l2(S64, U_ic)}
    accuracy["note"] = ("relative L2 over all GLL values, per conserved field (rho, rho u, rho v, rho w, E); "
                        "rho w starts at exactly zero, so its own relative figure compares round-off with a "
                        "near-zero norm: 'momentum_vector' takes the three momenta as one field and "
                        "'rho_w_vs_momentum_norm' measures the z-momentum error against that field's norm")

    # ---- end to end through the C ABI with pinned host buffers, both forms
    e2e = {name: measure_e2e(dgm_b200, doms[name], streams[name], prec, mesh, local, tiles[name]["variant"], dt,
                             args, barrier, max_over_ranks, world, dof)
           for name, prec in forms_run}

    peak, kind = peaks()
    fp64_peak = None
    try:
        fp64_peak = dgm_b200.fma_peak(True, local)
    except Exception:
        pass
    stage_mx, stage_64 = tmx / (14 * args.steps), t64 / (14 * args.steps)

    def roof(prec, stage_s, prof):
        a = BYTES_PER_DOF_STAGE[prec] * dof / stage_s / 1e9
        return {"bound": "hbm", "achieved": a, "peak": peak, "unit": "GB/s", "frac": a / peak,
                "peak_kind": kind, "traffic": profile_traffic(prof),
                "kernel": f"{tiles[prec]['kernel']}<Euler3D, L=4, Q=5, {prec}> (one launch per LSRK stage)",
                "algorithmic_bytes_per_launch": BYTES_PER_DOF_STAGE[prec] * dof,
                "stage_us": 1e6 * stage_s}

    fp64_roof = roof("fp64", stage_64, "euler3d_tgv_p3_stage_kernel.md")
    fp64_pipe = None
    if fp64_peak:
        ach = FLOPS_PER_DOF_STAGE * dof / stage_64 / 1e12
        fp64_pipe = {"bound": "fp64", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s", "frac": ach / fp64_peak,
                     "peak_kind": "measured live (dgmx_measure_fma_peak: FP64 FMA chains over a full grid)",
                     "algorithmic_flops_per_dof_stage": FLOPS_PER_DOF_STAGE}
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tmx / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 solution register)",
           "data": "synthetic (Taylor-Green initial condition, no dataset)",
           "config": config_dict(n, p, q, dof, world, "replicas"),
           "precision": "mixed: FP32 states, fluxes and contractions, FP64 solution register",
           "tile": tiles["mixed"],
           "fp64": {"value": v64, "unit": UNIT, "ms_per_step": 1e3 * t64 / args.steps, "tile": tiles["fp64"],
                    "roofline": fp64_roof, "roofline_fp64_pipe": fp64_pipe, "e2e": e2e["fp64"]},
           "speedup_mixed_vs_fp64": value / v64,
           "accuracy": accuracy,
           "e2e": e2e["mixed"],
           "gpu_launches": int(launches), "clocks": clk.summary(),
           "roofline": roof("mixed", stage_mx, "euler3d_tgv_p3_stage_mixed.md")}
    for Dx in doms.values():
        Dx.close()
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        try:
            v, tc = cpu_measure(n, p, q, 1, threads)
            out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                                   "sample": f"1 LSRK14 step (14 stages) of the full workload, FP64, {tc:.1f} s"}
        except Exception as ex:  # the baseline never blocks the GPU number
            out["cpu_baseline"] = {"value": None, "error": str(ex)[:200]}
    if rank == 0 and world == 1 and not args.no_forms:
        out["forms"] = forms(dgm_b200, args)
        out["other_configs"] = other_configs(dgm_b200, args)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
