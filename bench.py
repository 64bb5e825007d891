"""Benchmark of the SIMPLE pressure-velocity path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|mixed] [--cells NXxNYxNZ]

Workload (one GPU): steady SIMPLE on the 3-D channel of 128 x 64 x 64 hex cells
(524,288 cells) on [0,4]x[0,1]x[0,1], interior nodes jittered +-10 % (seed 0),
cells shuffled then renumbered by reverse Cuthill-McKee; parabolic inlet
(Umean = 1), pressure outlet, no-slip walls, rho = 1, mu = 5e-3; BiCGStab+Jacobi
on momentum and PCG+ILU(0) on the pressure correction, both to 1e-8 relative.
A step is one SIMPLE outer iteration; `value` is outer iterations per second
over all ranks (weak scaling: one case per GPU).

`--impl reference` times the CPU restatement of the reference's serial
simple_run (the oracle, one thread: the reference's serial solver has no
threading) on the same workload and prints the same line with impl=reference.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SIMPLE outer iters/s & p99 solve latency, mixed vs FP64 GPU at 1e-8 rel L2"
UNIT = "outer_iters/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--cells", default="128x64x64")
    ap.add_argument("--lin-max", type=int, default=1000)
    ap.add_argument("--cpu-steps", type=int, default=2, help="oracle outer iterations for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload(args, order_fn):
    from mixsolver_b200 import abi, cases
    nx, ny, nz = (int(v) for v in args.cells.split("x"))
    mesh, ctrl = cases.channel3d(nx, ny, nz, seed=0, outer_max=10 ** 6, order_fn=order_fn,
                                 mom=abi.MOM_JACOBI, ppe=abi.PPE_ILU0)
    ctrl.lin_max = args.lin_max
    ctrl.precision = abi.PREC_MIXED if args.precision == "mixed" else abi.PREC_FP64
    return mesh, ctrl


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8 for i in range(4)
                          if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def krylov_bytes(n, nnz, its, method):
    """Algorithmic bytes of one Krylov solve (unique footprint per operation):
    SpMV 12 nnz + 4(N+1) + 16 N; triangular pair 12 nnz + 24 N; dot 16 N;
    axpy 24 N; norm 8 N; Jacobi apply 20 N."""
    spmv = 12 * nnz + 4 * (n + 1) + 16 * n
    tri = 12 * nnz + 24 * n
    jac = 20 * n
    if method == "pcg":   # per iteration: SpMV, p.q, 2 axpy, norm, apply, r.z, p update
        per = spmv + 16 * n + 48 * n + 8 * n + tri + 16 * n + 24 * n
        setup = spmv + 8 * n + 8 * n + 12 * nnz  # b norm, r = b - Ax, factor copy
    else:                 # BiCGStab-Jacobi: 2 SpMV, 2 applies, 6 reductions, 5 updates
        per = 2 * spmv + 2 * jac + 16 * n * 3 + 8 * n * 2 + 16 * n + 24 * n * 4 + 8 * n
        setup = spmv + 8 * n + 24 * n
    return setup + its * per


def run_ours(args):
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    from mixsolver_b200 import solver as S
    mesh, ctrl = workload(args, S.rcm_order)
    case = S.UnsCase(mesh, ctrl, device=local)
    N, F = mesh.ncells, mesh.nfaces
    nnz = N + 2 * mesh.n_interior()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
    # warm-up
    ier, _ = case.simple_run(args.warmup)
    assert ier == 0, f"warm-up ier={ier}"
    case.set_profiling(True)
    barrier()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        ier, log = case.simple_run(args.steps, logcap=args.steps)
        wall = time.perf_counter() - t0
    barrier()
    assert ier == 0 and len(log) == args.steps, (ier, len(log))
    tm = case.timing()
    dev_ms = tm["total_ms"]
    mx = dev_ms
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([dev_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        mx = float(t.item())
    value = world * args.steps / (mx / 1e3)
    # roofline of the dominant kernel family (Krylov solves; factor + solve per launch pair)
    its_mom = sum(sum(r["lin_it"][:3]) for r in log)
    its_ppe = sum(r["lin_it"][3] for r in log)
    kbytes = (sum(krylov_bytes(N, nnz, r["lin_it"][c], "bicg") for r in log for c in range(3)) +
              sum(krylov_bytes(N, nnz, r["lin_it"][3], "pcg") for r in log))
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    kms = tm["krylov_ms"]
    nk = max(1, tm["krylov_launches"])
    achieved = kbytes / (kms / 1e3) / 1e9 if kms > 0 else None
    # end to end through the public API: host fields in, one outer iteration, fields out
    u = np.ascontiguousarray(case.fields()["u"])
    h2d = (3 * N + N + F) * 8
    d2h = (3 * N + N + F) * 8
    f = case.fields()
    barrier()
    e2e_steps = max(2, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        case.upload(u=f["u"], p=f["p"], flux=f["flux"])
        ier, _ = case.simple_run(1, logcap=1)
        f = case.fields()
    e2e_t = time.perf_counter() - t0
    e2e = {"value": world * e2e_steps / e2e_t, "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h + 9 * 8 * N + 8 * N + 3 * 8 * N}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mx / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32-inner/f64",
        "data": "synthetic (seeded jittered hex channel, RCM-ordered)",
        "config": {"workload": f"steady SIMPLE, 3-D channel {args.cells} hex ({N} cells), "
                               "BiCGStab+Jacobi momentum, PCG+ILU(0) pressure, lin_tol 1e-8",
                   "cells": N, "faces": F, "nnz": nnz, "lin_max": args.lin_max,
                   "precision": args.precision, "parallelism": f"replicas x{world}",
                   "l2": "working set per outer iteration ~0.4 GB > 126 MB L2 (no explicit flush)",
                   "krylov_iterations_per_step": {"momentum": its_mom / args.steps, "pressure": its_ppe / args.steps}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": None,
                     "kernel": "persistent Krylov solves (factor + solve per launch pair)",
                     "launches": nk, "avg_launch_ms": kms / nk, "peak_source": "MEASURED_PEAKS.json hbm_gbs"},
        "e2e": e2e,
        "gpu_launches": tm["gpu_launches"],
        "clocks": clk.summary(),
        "wall_s": wall,
    }
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args, mesh, ctrl)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def cpu_baseline(args, mesh, ctrl, steps=None):
    """The oracle (CPU restatement of the reference's serial simple_run, one
    thread) on the same mesh and control, timed over a few outer iterations."""
    from oracle import oracle as O
    steps = steps or args.cpu_steps
    oc = O.OracleCase(mesh, ctrl)
    t0 = time.perf_counter()
    ier, log = oc.simple_run(steps)
    dt = time.perf_counter() - t0
    return {"value": steps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{steps} outer iterations of the same {mesh.ncells}-cell channel from rest, "
                      f"{dt:.1f} s, pressure iterations {[r['lin_it'][3] for r in log]}"}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return
    # the same input mesh as the GPU arm: reverse Cuthill-McKee order (restated in oracle/rcm.py)
    from oracle import oracle as O
    from oracle.rcm import rcm
    mesh, ctrl = workload(args, rcm)
    oc = O.OracleCase(mesh, ctrl)
    w = min(args.warmup, 1)
    k = max(1, min(args.steps, 3))
    oc.simple_run(w)
    t0 = time.perf_counter()
    ier, log = oc.simple_run(k)
    dt = time.perf_counter() - t0
    value = k / dt
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": k, "warmup": w,
           "ms_per_step": 1e3 * dt / k, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded jittered hex channel, RCM-ordered)", "impl": "reference",
           "config": {"workload": f"steady SIMPLE, 3-D channel {args.cells} hex ({mesh.ncells} cells), "
                                  "BiCGStab+Jacobi momentum, PCG+ILU(0) pressure, lin_tol 1e-8",
                      "cells": mesh.ncells, "lin_max": args.lin_max},
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                            "sample": f"{k} outer iterations after {w} warm-up (steps capped at 3 to bound "
                                      "the CPU run); the reference's serial SIMPLE is single-threaded"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)
