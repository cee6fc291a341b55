#!/usr/bin/env python3
"""DOF-stage-updates/s of the B200 DG engine on the 3-D Euler Taylor-Green case.

Workload (the single-GPU configuration the metric is quoted on): periodic
[0, 2pi]^3, 32^3 Hex elements, p = 3 (q = 5 GLL points per direction),
compressible Euler, Lax-Friedrichs flux, low-storage RK (LSRK14, 14 stages),
Mach 0.1 Taylor-Green initial condition, FP64.  dt is fixed once from CFL 0.5
on the initial state.  A "step" is one LSRK14 step (14 fused stage launches).

  value  device-resident throughput: modal DOF x 14 stages x K / time (CUDA
         events on the engine's stream, max over ranks)
  e2e    the same metric through the public C ABI with host buffers: every
         step uploads the state from pinned host memory (dgmx_set_state),
         advances one step (dgmx_advance) and reads the state back
         (dgmx_get_state)
Ranks (torchrun, N > 1) run independent replicas of the workload (weak
scaling, no collective in the data path; NCCL only for the barrier and the
max-over-ranks time).  --impl reference times the CPU restatement of the
reference algorithm (the oracle) on the host cores instead.
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

WORKLOAD = dict(name="euler3d_taylor_green_32^3_p3_lsrk14", n=32, p=3, q=5, Ma=0.1, gamma=1.4, cfl=0.5)
METRIC = "DOF-stage-updates/s"
BYTES_PER_DOF_STAGE = 32  # read U, read Ut, write Ut, write U (FP64)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--n", type=int, default=WORKLOAD["n"], help="elements per direction")
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


def profile_traffic():
    """DRAM bytes per stage launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "euler3d_tgv_p3_stage_kernel.md")
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
    return oracle.Problem(mesh, oracle.EULER3D)


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


def config_dict(n, p, q, dof):
    return {"workload": WORKLOAD["name"] if n == WORKLOAD["n"] else f"euler3d_taylor_green_{n}^3_p{p}_lsrk14",
            "mesh": f"{n}^3 Hex, periodic [0,2pi]^3", "p": p, "q": q, "physics": "Euler 3-D",
            "flux": "Lax-Friedrichs", "integrator": "LSRK14 (14 stages/step)", "Mach": WORKLOAD["Ma"],
            "modal_dof": dof, "cfl": WORKLOAD["cfl"],
            "l2": "inputs larger than L2 (modal U+Ut 168 MB, traces 2x126 MB per replica)"}


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
    out = {"metric": METRIC, "value": v, "unit": "DOF-stage-updates/s", "impl": "reference",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (Taylor-Green initial condition)", "config": config_dict(n, p, q, dof),
           "cpu_baseline": {"value": v, "unit": "DOF-stage-updates/s", "cores": threads, "kind": "port",
                            "sample": f"{args.steps} LSRK14 steps of the full workload after {args.warmup} warm-up"},
           "e2e": {"value": v, "unit": "DOF-stage-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)
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
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    n, p, q = args.n, WORKLOAD["p"], WORKLOAD["q"]
    mesh = dgm_b200.meshgen.box(3, (n, n, n), 0.0, 2 * math.pi, p, q)
    D = dgm_b200.Domain(mesh, dgm_b200.EULER3D, flux="laxfriedrichs", inttype=dgm_b200.LSRK14, device=local)
    x, y, z = D.coordinates()
    U_ic = taylor_green(x, y, z, WORKLOAD["Ma"], WORKLOAD["gamma"])
    D.set_state(U_ic)
    dt = cfl_dt(U_ic, 2 * math.pi / n, p, WORKLOAD["gamma"], WORKLOAD["cfl"])
    dof = 5 * n ** 3 * (p + 1) ** 3
    stream = torch.cuda.ExternalStream(D.stream(), device=torch.device("cuda", local))
    # tile autotuning is set-up, outside the timed region
    tune_rows, tune_pick = D.autotune(reps=10)
    tile = {"elements_per_cta": int(tune_rows[tune_pick][0]), "min_ctas_per_sm": int(tune_rows[tune_pick][1]),
            "threads_per_cta": int(tune_rows[tune_pick][2]),
            "candidates_us": [round(float(r[3]), 1) for r in tune_rows]}

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

    # ---- device-resident fused LSRK14 steps
    for _ in range(args.warmup):
        D.advance_async(dt, 1)
    D.sync()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = D.launch_count()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            D.advance_async(dt, 1)
        ev1.record(stream)
        ev1.synchronize()
    launches = D.launch_count() - l0
    D.sync()
    barrier()
    t = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    value = world * dof * 14 * args.steps / t
    stage_s = t / (14 * args.steps)

    # ---- end to end through the C ABI with pinned host buffers
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
    e2e = world * dof * 14 * ke / te
    nbytes = 5 * D.nq * 8

    out = {"metric": METRIC, "value": value, "unit": "DOF-stage-updates/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (Taylor-Green initial condition, no dataset)",
           "config": config_dict(n, p, q, dof) | {"parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                                                  "tile": tile},
           "e2e": {"value": e2e, "unit": "DOF-stage-updates/s", "h2d_bytes_per_step": nbytes,
                   "d2h_bytes_per_step": nbytes, "steps": ke,
                   "path": "dgmx_set_state + dgmx_advance(1 step) + dgmx_get_state, pinned host buffers"},
           "gpu_launches": int(launches), "clocks": clk.summary()}
    peak, kind = peaks()
    achieved = BYTES_PER_DOF_STAGE * dof / stage_s / 1e9
    out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                       "frac": achieved / peak, "peak_kind": kind, "traffic": profile_traffic(),
                       "kernel": "stage_kernel<Euler3D, L=4, Q=5> (one launch per LSRK stage)",
                       "algorithmic_bytes_per_launch": BYTES_PER_DOF_STAGE * dof}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        try:
            v, tc = cpu_measure(n, p, q, 1, threads)
            out["cpu_baseline"] = {"value": v, "unit": "DOF-stage-updates/s", "cores": threads, "kind": "port",
                                   "sample": f"1 LSRK14 step (14 stages) of the full workload, {tc:.1f} s"}
        except Exception as ex:  # the baseline never blocks the GPU number
            out["cpu_baseline"] = {"value": None, "error": str(ex)[:200]}
    if rank == 0:
        print(json.dumps(out), flush=True)
    D.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
