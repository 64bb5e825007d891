"""Benchmark of the SIMPLE pressure-velocity path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision fp64|mixed] [--cells NXxNYxNZ]
                    [--workload channel|batch|serve|piso|pimple]

Workload (one GPU): steady SIMPLE on the 3-D channel of 128 x 64 x 64 hex cells
(524,288 cells) on [0,4]x[0,1]x[0,1], interior nodes jittered +-10 % (seed 0),
cells shuffled then renumbered by reverse Cuthill-McKee; parabolic inlet
(Umean = 1), pressure outlet, no-slip walls, rho = 1, mu = 5e-3; linear solves
to 1e-8 relative. A step is one SIMPLE outer iteration; `value` is outer
iterations per second over all ranks (weak scaling: one case per GPU).

The measured form (--precision, default mixed) is the mixed-precision one;
the FP64 parity form (BiCGStab+Jacobi momentum, PCG+ILU(0) pressure, the
reference's arithmetic) runs the same outer iterations beside it, and the
line reports its rate and the relative L2 difference of u, p, flux.

The other workloads print their own lines: `batch` (many 3-D cavities in one
batched iteration), `serve` (a Poisson stream of SIMPLE / PISO requests with
p50 / p99 latency), `piso` (80^3 x 6 tets, transient) and `pimple` (the
reference's 80 x 80 x 1 cavity PIMPLE run, against its published step time).

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
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--cells", default="128x64x64")
    ap.add_argument("--lin-max", type=int, default=1000)
    ap.add_argument("--cpu-steps", type=int, default=2, help="oracle outer iterations for cpu_baseline")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="channel", choices=["channel", "batch", "serve", "piso", "pimple"],
                    help="channel: one 524k-cell case (default); batch: many 3-D cavities in one batch; "
                         "serve: a Poisson stream of SIMPLE / PISO requests; piso: transient PISO on "
                         "80^3 x 6 tets; pimple: transient PIMPLE on the 80 x 80 x 1 lid-driven cavity")
    ap.add_argument("--tet-n", type=int, default=80, help="piso: hexes per cube edge (each split into 6 tets)")
    ap.add_argument("--fp64-steps", type=int, default=3, help="piso: time steps of the FP64 comparison leg")
    ap.add_argument("--rate", type=float, default=50.0, help="serve: arrivals per second")
    ap.add_argument("--duration", type=float, default=2.0, help="serve: seconds of arrivals (mixed leg)")
    ap.add_argument("--fp64-duration", type=float, default=0.5, help="serve: seconds of arrivals (FP64 leg)")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="serve: device memory for resident cases")
    ap.add_argument("--active-cells", type=int, default=4_000_000, help="serve: cells stepped together per tick")
    ap.add_argument("--cases", type=int, default=256, help="batch: number of cavity cases")
    ap.add_argument("--policy", default="auto", help="batch: lane policy SPLIT_ROWSxWIDE_LANES or auto")
    ap.add_argument("--fp64-iters", type=int, default=2, help="batch: iterations of the FP64 comparison leg")
    ap.add_argument("--accuracy-iters", type=int, default=200,
                    help="channel: outer iterations after which the mixed form is compared with the tight FP64 run")
    ap.add_argument("--tight-tol", type=float, default=1e-12, help="channel: lin_tol of the tight FP64 run")
    ap.add_argument("--tuning", default="",
                    help="library tuning keys set before the run (mgpu_set_tuning), e.g. ell_stage=0,cheb_degree=12")
    return ap.parse_args()


def apply_tuning(args):
    """Set the --tuning keys; returns them as a dict for the config record."""
    from mixsolver_b200 import solver as S
    out = {}
    for kv in filter(None, args.tuning.split(",")):
        k, v = kv.split("=")
        S.set_tuning(k.strip(), int(v))
        out[k.strip()] = int(v)
    return out


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_ranks(world, backend="nccl", timeout_s=600):
    """One process per GPU: the process group of a run with world > 1 ranks
    (rendezvous from MASTER_ADDR / MASTER_PORT); nothing for one rank."""
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))


def rank_barrier(world, cuda=True):
    """Device idle on this rank, then every rank at the same point."""
    import torch
    if cuda:
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v, world, device="cuda"):
    """The largest of the ranks' values (device times are taken as the max)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, world, max_ms):
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return world * units_per_rank / (max_ms / 1e3)


def close_ranks(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


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
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a moment to start: wait (at most 2 s) for its first
            # row, so a short timed region still gets samples
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 2.0 and self.proc.poll() is None:
                time.sleep(0.01)
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


def pinned_fields(case):
    """Page-locked host arrays for every field of ``case`` (UnsCase.fields(out=...))."""
    import torch
    dims = {"N": case.N, "F": case.F}
    return {k: torch.empty(tuple(dims.get(d, d) for d in shp), dtype=torch.float64, pin_memory=True).numpy()
            for k, shp in case.FIELD_SHAPES.items()}


def hbm_peak():
    """The roofline denominator: the measured HBM copy rate of this pool's B200s
    (MEASURED_PEAKS.json, "of measured"), else the earlier measurement of
    6.65 TB/s ("of fallback")."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        v = float(json.load(open(path))["hbm_gbs"])
        return v, "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except (OSError, ValueError, KeyError, TypeError):
        return 6650.0, "6.65 TB/s earlier measurement on this pool (of fallback)"


def krylov_bytes(n, nnz, its, method, mixed=False, tol=1e-8, tau=1e-4, cheb_k=None):
    """Algorithmic bytes of one Krylov solve: the unique footprint of every
    pass over the system (matrix entries once, each vector read or written
    once per pass), in the solver's own arithmetic types.

    FP64 form: SpMV 12 nnz + 4(N+1) + 16 N; triangular pair 12 nnz + 24 N;
    dot 16 N; axpy 24 N; norm 8 N; Jacobi apply 20 N.
    Mixed form:
      PCG: FP64 conjugate gradients with an FP32 degree-k Chebyshev-Jacobi
      polynomial, per iteration:
        p = z + beta p, q = A p (FP64 values + int32 columns = 12 B per
        entry; z FP32, p FP64), p.q:                          12 nnz + 28 N
        x += alpha p, r -= alpha q (FP64), FP32 copy of r and
        the first Chebyshev term:                              60 N
        k - 1 Chebyshev steps in FP32 (FP32 values + int32
        columns = 8 B per entry), each an SpMV plus 5 vectors: 8 nnz + 24 N
        (the last one also reads the FP64 r for r.z:            + 8 N)
      plus the prologue (FP32 and FP64 ELL copies of A: 8 + 12 + 8 nnz from
      12 nnz) and two FP64 true residuals (12 nnz + 4(N+1) + 28 N).
      BiCGStab-Jacobi (FP32 inside FP64 refinement), per iteration: 2 SpMV
      (8 nnz + 4(N+1) + 8 N) + 80 N; plus the prologue (FP32 copy of A:
      12 nnz) and, per refinement step, one FP64 true residual and the x
      update."""
    import math
    if cheb_k is None:  # the degree the library runs with for n rows (the cheb_* tuning keys)
        from mixsolver_b200 import solver as S
        big = S.get_tuning("cheb_large_rows")
        cheb_k = S.get_tuning("cheb_degree_large" if 0 < big <= n else "cheb_degree")
    if mixed:
        true_res = 12 * nnz + 4 * (n + 1) + 28 * n
        if method == "pcg":
            setup = 40 * nnz + 24 * n + 2 * true_res + 28 * n
            per = (12 * nnz + 28 * n) + 60 * n + max(0, cheb_k - 1) * (8 * nnz + 24 * n) + 8 * n
            return setup + its * per
        steps = max(1, math.ceil(math.log(tol) / math.log(tau)))
        setup = 12 * nnz + 24 * n + steps * (true_res + 28 * n + 20 * n)
        per = 2 * (8 * nnz + 4 * (n + 1) + 8 * n) + 80 * n
        return setup + its * per
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


def channel_config(args, mesh):
    """The workload's `config`, the same dict in both arms."""
    N, F = mesh.ncells, mesh.nfaces
    return {"workload": f"steady SIMPLE, 3-D channel {args.cells} hex ({N} cells), jittered, RCM order; "
                        f"lin_tol 1e-8; {args.warmup} warm-up + {args.steps} timed outer iterations from rest",
            "cells": N, "faces": F, "nnz": N + 2 * mesh.n_interior(), "lin_tol": 1e-8, "lin_max": args.lin_max,
            "parallelism": "one case per rank (replicas)",
            "l2": "each outer iteration touches ~0.45 GB of case arrays (> 126 MB L2): no explicit flush; "
                  "inside the pressure solve the FP32 system (~44 MB) stays in L2 across its passes"}


def l2_copy_gbs(device="cuda"):
    """Read+write rate of L2-resident element-wise traffic: c = a + b over
    three 16 MiB buffers (48 MiB, inside the 126 MB L2), 100 launches replayed
    from a CUDA graph so launch gaps do not count, timed with CUDA events: the
    L2 counterpart of the HBM copy peak, measured in the same run."""
    import torch
    n = 4 * 2 ** 20
    a = torch.ones(n, device=device)
    b = torch.ones(n, device=device)
    c = torch.empty(n, device=device)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(5):
            torch.add(a, b, out=c)
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(100):
            torch.add(a, b, out=c)
    g.replay()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    g.replay()
    e1.record()
    torch.cuda.synchronize()
    return 100 * 3 * n * 4 / (e0.elapsed_time(e1) / 1e3) / 1e9


def rel_fields(f, ref):
    return {k: float(np.linalg.norm(f[k] - ref[k]) / np.linalg.norm(ref[k])) for k in ("u", "p", "flux")}


def run_ours(args):
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    init_ranks(world)
    import copy
    from mixsolver_b200 import abi
    from mixsolver_b200 import solver as S
    mesh, ctrl = workload(args, S.rcm_order_device)  # cells renumbered by RCM on the device
    N, F = mesh.ncells, mesh.nfaces
    nnz = N + 2 * mesh.n_interior()
    mixed = args.precision == "mixed"
    W, K = args.warmup, args.steps
    A = max(args.accuracy_iters, W + K)

    barrier = lambda: rank_barrier(world)
    ranks_max = lambda v: max_over_ranks(v, world)

    def form(prec, tol=None, lin_max=None):
        c = copy.deepcopy(ctrl)
        c.precision = prec
        if tol is not None:
            c.lin_tol, c.lin_max = tol, lin_max
        return S.UnsCase(mesh, c, device=local)

    def rate_leg(prec):
        """W warm-up + K timed outer iterations from rest: rate, fields after W + K."""
        k = form(prec)
        ier, _ = k.simple_run(W)
        assert ier == 0
        barrier()
        ier, log = k.simple_run(K, logcap=K)
        barrier()
        assert ier == 0
        t = ranks_max(k.timing()["total_ms"])
        out = dict(value=job_rate(K, world, t), fields=k.fields(),
                   ppe_its=float(np.mean([r["lin_it"][3] for r in log])))
        k.close()
        return out

    fp64 = poly = tight = None
    if mixed:
        # the FP64 parity form (the reference's arithmetic) and the same solvers
        # as the mixed form in FP64 throughout (the FP32 gain alone)
        fp64 = rate_leg(abi.PREC_FP64)
        poly = rate_leg(abi.PREC_FP64_POLY)
        # the converged answer of the same outer iterations: FP64 solves to 1e-12,
        # in the same run segments as the measured case (W, K, then A - W - K)
        kt = form(abi.PREC_FP64_POLY, tol=args.tight_tol, lin_max=4000)
        tight = {}
        for seg, n_it in (("w", W), ("wk", K), ("a", A - W - K)):
            if n_it > 0:
                ier, _ = kt.simple_run(n_it)
                assert ier == 0
            tight[seg] = kt.fields()
        kt.close()
    case = S.UnsCase(mesh, ctrl, device=local)
    ier, _ = case.simple_run(W)
    assert ier == 0, f"warm-up ier={ier}"
    case.set_profiling(True)
    barrier()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        ier, log = case.simple_run(K, logcap=K)
        wall = time.perf_counter() - t0
    barrier()
    assert ier == 0 and len(log) == K, (ier, len(log))
    tm = case.timing()
    mx = ranks_max(tm["total_ms"])
    value = job_rate(K, world, mx)
    solve_ms = case.solve_times()
    ppe_ms = solve_ms[3::4] if len(solve_ms) >= 4 else solve_ms
    pct = lambda a, q: float(np.percentile(a, q)) if len(a) else None
    its_mom = sum(sum(r["lin_it"][:3]) for r in log)
    its_ppe = sum(r["lin_it"][3] for r in log)
    kb = lambda r, c, meth: krylov_bytes(N, nnz, r["lin_it"][c], meth, mixed, ctrl.lin_tol, ctrl.mixed_tol)
    kbytes = sum(kb(r, c, "bicg") for r in log for c in range(3)) + sum(kb(r, 3, "pcg") for r in log)
    peak, peak_source = hbm_peak()
    kms = tm["krylov_ms"]
    # the dominant kernel: the persistent pressure solve (one launch per outer
    # iteration), its algorithmic bytes over its CUDA-event time
    ppe_bytes = [kb(r, 3, "pcg") for r in log]
    ppe_launch_ms = float(np.mean(ppe_ms)) if len(ppe_ms) else None
    achieved = (float(np.mean(ppe_bytes)) / (ppe_launch_ms / 1e3) / 1e9) if ppe_launch_ms else None
    family = kbytes / (kms / 1e3) / 1e9 if kms > 0 else None
    f = case.fields()
    accuracy = None
    if mixed:
        f_wk = f
        if A > W + K:
            ier, _ = case.simple_run(A - W - K)
            assert ier == 0
        f_a = case.fields()
        accuracy = {
            "reference": f"the same outer iterations with every linear system solved in FP64 to lin_tol "
                         f"{args.tight_tol:g} (FP64 Chebyshev-Jacobi PCG / BiCGStab-Jacobi)",
            "mixed_vs_tight": {str(W + K): rel_fields(f_wk, tight["wk"]), str(A): rel_fields(f_a, tight["a"])},
            "fp64_form_vs_tight": {str(W + K): rel_fields(fp64["fields"], tight["wk"])},
            "mixed_vs_fp64_form": {str(W + K): rel_fields(f_wk, fp64["fields"])},
            "fp64_poly_vs_tight": {str(W + K): rel_fields(poly["fields"], tight["wk"])},
        }
        # the run's end state for the e2e leg below is the timed state's successor
        f = f_a
    # end to end through the public API: host fields in (page-locked), one outer
    # iteration and the fields out into page-locked arrays in one call
    # (mgpu_simple_run_fields: gp, gu and apc copied while the pressure solve runs)
    h2d = (3 * N + N + F) * 8
    d2h = (3 * N + N + F + 3 * N + 9 * N + N) * 8
    hbuf = pinned_fields(case)
    for k in ("u", "p", "flux"):
        hbuf[k][...] = f[k]
    barrier()
    e2e_steps = max(2, min(K, 5))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        case.upload(u=hbuf["u"], p=hbuf["p"], flux=hbuf["flux"])
        ier, _, _ = case.simple_run_fields(1, out=hbuf, logcap=1)
    e2e_t = max_over_ranks(time.perf_counter() - t0, world)
    e2e = {"value": world * e2e_steps / e2e_t, "unit": UNIT, "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h}
    l2peak = l2_copy_gbs()
    gate = accuracy["mixed_vs_tight"][str(A)] if accuracy else None
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": mx / K, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if not mixed else "f32-inner/f64-refinement",
        "data": "synthetic (seeded jittered hex channel, RCM-ordered)",
        "config": channel_config(args, mesh),
        "form": ("mixed: FP32 BiCGStab-Jacobi momentum inside FP64 refinement; pressure PCG in FP64 with an "
                 "FP32 Chebyshev-Jacobi polynomial preconditioner (FP32 matrix copy and vectors); every dot "
                 "product and norm FP64"
                 if mixed else "FP64 parity form: BiCGStab+Jacobi momentum, PCG+ILU(0) pressure"),
        "krylov_iterations_per_step": {"momentum": its_mom / K, "pressure": its_ppe / K},
        "solve_latency_ms": {"p50": pct(solve_ms, 50), "p99": pct(solve_ms, 99),
                             "pressure_p50": pct(ppe_ms, 50), "pressure_p99": pct(ppe_ms, 99)},
        "fp64_form": None if fp64 is None else {
            "outer_iters_per_s": fp64["value"], "pressure_iterations_per_step": fp64["ppe_its"],
            "solvers": "BiCGStab+Jacobi momentum, PCG+ILU(0) pressure (exact, parity form)"},
        "fp64_poly_form": None if poly is None else {
            "outer_iters_per_s": poly["value"], "pressure_iterations_per_step": poly["ppe_its"],
            "solvers": "the mixed form's solvers in FP64 throughout"},
        "speedup_vs_fp64": None if fp64 is None else value / fp64["value"],
        "speedup_vs_fp64_poly": None if poly is None else value / poly["value"],
        "rel_l2_vs_fp64": None if gate is None else dict(
            gate, against=f"FP64 solved to lin_tol {args.tight_tol:g}, after {A} outer iterations"),
        "accuracy": accuracy,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     # DRAM bytes of one pressure-solve launch (36 iterations at the default
                     # degree 24) from an ncu capture of this workload
                     # (profiles/k_pcg_mixed_channel524k.md)
                     "traffic": 1.914e9 if mixed and S.get_tuning("cheb_degree") == 24 else None,
                     "resident": "L2: the system (~94 MB with its FP64 copy) stays in the 126 MB L2 across the "
                                 "solve's passes, DRAM carries 5 % of the algorithmic bytes (ncu); frac is an "
                                 "HBM-equivalent rate, see l2 for the fraction of the L2 roofline",
                     "l2": {"achieved": achieved, "peak": l2peak, "unit": "GB/s",
                            "frac": (achieved / l2peak) if achieved else None,
                            "peak_source": "L2-resident c = a + b over 3 x 16 MiB buffers, graph-replayed, "
                                           "measured in this run"},
                     "kernel": "k_pcg_mixed (pressure solve)" if mixed else "k_factor+k_pcg (pressure solve)",
                     "algorithmic_bytes_per_launch": float(np.mean(ppe_bytes)), "avg_launch_ms": ppe_launch_ms,
                     "launches": len(ppe_ms), "all_krylov_solves_gbs": family,
                     "peak_source": peak_source},
        "e2e": e2e,
        "gpu_launches": tm["gpu_launches"],
        "clocks": clk.summary(),
        "wall_s": wall,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:  # the CPU baseline is an N = 1 figure
        out["cpu_baseline"] = cpu_baseline(args, mesh, ctrl)
    close_ranks(world)
    if rank == 0:
        if getattr(args, "tuning_set", None):
            out["config"]["tuning"] = args.tuning_set
        print(json.dumps(out), flush=True)


def cpu_baseline(args, mesh, ctrl, steps=None):
    """The oracle (CPU restatement of the reference's serial simple_run, one
    thread) on the same mesh and control, timed over a few outer iterations.
    The reference's solvers for this workload are the FP64 ones."""
    import copy
    from mixsolver_b200 import abi
    from oracle import oracle as O
    steps = steps or args.cpu_steps
    ctrl = copy.deepcopy(ctrl)
    ctrl.precision = abi.PREC_FP64
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
    # the same outer iterations as the GPU arm's timed region (about 4-6 s each
    # on one core): W warm-up and K timed, each capped (5 and 20) to bound the run
    w = min(args.warmup, 5)
    k = max(1, min(args.steps, 20))
    oc.simple_run(w)
    t0 = time.perf_counter()
    ier, log = oc.simple_run(k)
    dt = time.perf_counter() - t0
    value = k / dt
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0, "steps": k, "warmup": w,
           "ms_per_step": 1e3 * dt / k, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic (seeded jittered hex channel, RCM-ordered)", "impl": "reference",
           "config": channel_config(args, mesh),
           "form": "the reference's serial simple_run restated (oracle): BiCGStab+Jacobi momentum, "
                   "PCG+ILU(0) pressure, FP64",
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                            "sample": f"outer iterations {w + 1}..{w + k} after {w} warm-up (the GPU arm's timed "
                                      "iterations when W <= 5 and K <= 20); the reference's serial SIMPLE is "
                                      "single-threaded"},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


PISO_METRIC = "PISO time steps/s, mixed vs FP64 GPU, rel L2 of u, p vs FP64"
# DRAM bytes of the first corrector's pressure solve on the 3.07 M-tet box, by
# Chebyshev degree, from ncu captures (profiles/k_pcg_mixed_piso3M.md)
PISO_TRAFFIC = {24: 539.5e9, 48: 527.1e9}


def run_piso(args):
    """Transient PISO on n^3 unit-cube hexes each split into 6 tets (n = 80:
    3,072,000 tets), RCM-ordered, no-slip walls, rho = 1, mu = 1e-3, dt = 1e-3,
    2 correctors, implicit Euler, seeded Taylor-Green start (amplitude 1, 1 %
    uniform noise); linear solves to 1e-10 relative. A step is one time step.
    The mixed form (FP32 SpMV and preconditioner inside FP64 refinement) and
    the FP64 form (BiCGStab+Jacobi momentum, PCG+IC(0) pressure) first run the
    same --fp64-steps steps from the same start, and the line reports the
    relative L2 difference of u, p and flux after them; the mixed case then
    runs W warm-up and K timed steps."""
    rank, world, local = dist_env()
    import copy
    import torch
    torch.cuda.set_device(local)
    init_ranks(world)
    from mixsolver_b200 import abi, cases, meshgen
    from mixsolver_b200 import solver as S
    total = args.fp64_steps + args.warmup + args.steps
    mesh, ctrl = cases.tet_box(args.tet_n, steps=total + 8, ppe=abi.PPE_IC0, mom=abi.MOM_JACOBI)
    mesh = cases.rcm_renumber(mesh, S.rcm_order)
    ctrl.lin_tol = 1e-10
    ctrl.lin_max = args.lin_max
    N, F = mesh.ncells, mesh.nfaces
    nnz = N + 2 * mesh.n_interior()
    u0 = meshgen.taylor_green(S.compute_geometry(mesh)["xc"], seed=rank)

    barrier = lambda: rank_barrier(world)
    ranks_max = lambda v: max_over_ranks(v, world)

    def make(prec):
        c = copy.deepcopy(ctrl)
        c.precision = prec
        k = S.UnsCase(mesh, c, device=local)
        k.upload(u=u0)
        return k

    # FP64 comparison leg
    k64 = make(abi.PREC_FP64)
    ier, log64 = k64.piso_run(args.fp64_steps, logcap=args.fp64_steps)
    assert ier == 0, f"FP64 leg ier={ier}"
    t64 = ranks_max(k64.timing()["total_ms"])
    f64 = k64.fields()
    k64.close()
    # mixed form: the same steps, then warm-up and the timed steps
    case = make(abi.PREC_MIXED)
    ier, logc = case.piso_run(args.fp64_steps, logcap=args.fp64_steps)
    assert ier == 0, f"mixed comparison steps ier={ier}"
    fc = case.fields()
    rel = {k: float(np.linalg.norm(fc[k] - f64[k]) / np.linalg.norm(f64[k])) for k in ("u", "p", "flux")}
    t_cmp = ranks_max(case.timing()["total_ms"])
    if args.warmup:
        ier, _ = case.piso_run(args.warmup, logcap=args.warmup)
        assert ier == 0, f"warm-up ier={ier}"
    case.set_profiling(True)
    barrier()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        ier, log = case.piso_run(args.steps, logcap=args.steps)
        wall = time.perf_counter() - t0
    barrier()
    assert ier == 0 and len(log) == args.steps, (ier, len(log))
    tm = case.timing()
    mx = ranks_max(tm["total_ms"])
    value = job_rate(args.steps, world, mx)
    solve_ms = case.solve_times()
    nsol = 3 + ctrl.n_correct
    ppe_ms = np.concatenate([solve_ms[3 + j::nsol] for j in range(ctrl.n_correct)]) if len(solve_ms) >= nsol else solve_ms
    pct = lambda a, q: float(np.percentile(a, q)) if len(a) else None
    ppe_bytes = [krylov_bytes(N, nnz, r["lin_it"][3 + j], "pcg", True, ctrl.lin_tol, ctrl.mixed_tol)
                 for r in log for j in range(ctrl.n_correct)]
    kbytes = (sum(krylov_bytes(N, nnz, r["lin_it"][c], "bicg", True, ctrl.lin_tol, ctrl.mixed_tol)
                  for r in log for c in range(3)) + sum(ppe_bytes))
    peak, peak_source = hbm_peak()
    ppe_launch_ms = float(np.mean(ppe_ms)) if len(ppe_ms) else None
    achieved = (float(np.mean(ppe_bytes)) / (ppe_launch_ms / 1e3) / 1e9) if ppe_launch_ms else None
    family = kbytes / (tm["krylov_ms"] / 1e3) / 1e9 if tm["krylov_ms"] > 0 else None
    # end to end through the public API: host velocity in (page-locked), one time
    # step, fields out into page-locked arrays
    h2d = 3 * N * 8
    d2h = (3 * N + N + F + 3 * N + 9 * N + N) * 8
    hbuf = pinned_fields(case)
    case.fields(out=hbuf)
    barrier()
    e2e_steps = max(2, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        case.upload(u=hbuf["u"])
        ier, _ = case.piso_run(1, logcap=1)
        case.fields(out=hbuf)
    e2e_t = max_over_ranks(time.perf_counter() - t0, world)
    its = lambda lg, sl: float(np.mean([sum(r["lin_it"][c] for c in sl) for r in lg]))
    out = {
        "metric": PISO_METRIC, "value": value, "unit": "time_steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mx / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32-inner/f64-refinement",
        "data": "synthetic (seeded Taylor-Green start in a walled hex-split-tet box, RCM-ordered)",
        "config": {"workload": f"transient PISO, {args.tet_n}^3 x 6 tets ({N} cells), dt 1e-3, 2 correctors, "
                               "Euler, lin_tol 1e-10; mixed form: FP32-inner/FP64-refinement BiCGStab-Jacobi "
                               "and PCG with Chebyshev-Jacobi",
                   "cells": N, "faces": F, "nnz": nnz, "lin_max": args.lin_max, "parallelism": f"replicas x{world}",
                   "l2": "per-step working set > 126 MB L2 (no explicit flush)",
                   "krylov_iterations_per_step": {"momentum": its(log, range(3)),
                                                  "pressure": its(log, range(3, nsol))},
                   "solve_latency_ms": {"p50": pct(solve_ms, 50), "p99": pct(solve_ms, 99),
                                        "pressure_p50": pct(ppe_ms, 50), "pressure_p99": pct(ppe_ms, 99)},
                   "fp64_form": {"time_steps_per_s": world * args.fp64_steps / (t64 / 1e3),
                                 "steps": args.fp64_steps,
                                 "krylov_iterations_per_step": {"momentum": its(log64, range(3)),
                                                                "pressure": its(log64, range(3, nsol))},
                                 "solvers": "BiCGStab+Jacobi momentum, PCG+IC(0) pressure (parity form)"},
                   "mixed_comparison_steps_per_s": world * args.fp64_steps / (t_cmp / 1e3),
                   "speedup_vs_fp64": value / (world * args.fp64_steps / (t64 / 1e3)),
                   "rel_l2_vs_fp64": rel, "rel_l2_after_steps": args.fp64_steps},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     # DRAM bytes of one pressure-solve launch (the first corrector) from
                     # an ncu capture of this workload at the degree in effect
                     # (profiles/k_pcg_mixed_piso3M.md)
                     "traffic": PISO_TRAFFIC.get(S.get_tuning("cheb_degree_large")
                                                 if 0 < S.get_tuning("cheb_large_rows") <= N
                                                 else S.get_tuning("cheb_degree")),
                     "kernel": "k_pcg_mixed (pressure solves)",
                     "algorithmic_bytes_per_launch": float(np.mean(ppe_bytes)), "avg_launch_ms": ppe_launch_ms,
                     "launches": len(ppe_ms), "all_krylov_solves_gbs": family,
                     "peak_source": peak_source},
        "e2e": {"value": world * e2e_steps / e2e_t, "unit": "time_steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": tm["gpu_launches"],
        "clocks": clk.summary(),
        "wall_s": wall,
    }
    case.close()
    close_ranks(world)
    if rank == 0:
        if getattr(args, "tuning_set", None):
            out["config"]["tuning"] = args.tuning_set
        print(json.dumps(out), flush=True)


PIMPLE_METRIC = "PIMPLE time steps/s (FP64), 2-D lid-driven cavity Re 1000, 80 x 80 x 1"
PIMPLE_PUBLISHED_STEPS_PER_S = 1.0 / 0.182  # the reference's 6000-step run: 18.2 min, MPI np = 4


def pimple_case():
    """The reference's transient cavity run: 80 x 80 x 1 hex (zones 4 symmetry /
    5 wall, lid u = (1,0,0) on y = 1), rho = 1, mu = 1e-3 (Re 1000), dt = 0.01,
    2 outer iterations x 2 pressure corrections per step, alpha_u = 0.7,
    limited second-order upwind (conv_blend 1), no non-orthogonal correction,
    PCG+IC(0) pressure and BiCGStab+ILU(0) momentum to 1e-8 (lin_max 300)."""
    from mixsolver_b200 import abi, cases
    mesh, ctrl = cases.cavity2d(80, mu=1.0e-3, conv_blend=1.0, nonorth=0.0)
    ctrl.transient = True
    ctrl.dt = 0.01
    ctrl.n_time_max = 10 ** 6
    ctrl.n_outer_iter = 2
    ctrl.n_correct = 2
    ctrl.alpha_u = 0.7
    ctrl.lin_tol = 1e-8
    ctrl.lin_max = 300
    ctrl.ppe_precond = abi.PPE_IC0
    ctrl.mom_solver = abi.MOM_ILU0
    return mesh, ctrl


def run_pimple(args):
    """Transient PIMPLE (pimple_run_mpi at one rank) on the 80 x 80 x 1 cavity
    of :func:`pimple_case`, from rest, W warm-up and K timed time steps through
    mgpu_pimple_run; `value` in time steps per second over all ranks (one case
    per GPU). The measured form (--precision, default mixed: FP32 Krylov
    inside FP64 refinement to the same lin_tol) runs beside the FP64 parity
    form (the reference's arithmetic: exact IC(0)/ILU(0) sweeps), over the same
    steps; the line reports both rates and the relative L2 difference of u, p,
    flux after them. The reference publishes 0.182 s per step for this run
    (CPU, MPI np = 4), so `vs_baseline` is value / 5.49."""
    rank, world, local = dist_env()
    import copy
    import torch
    torch.cuda.set_device(local)
    init_ranks(world)
    from mixsolver_b200 import abi
    from mixsolver_b200 import solver as S
    mesh, ctrl = pimple_case()
    N, F = mesh.ncells, mesh.nfaces
    mixed = args.precision == "mixed"

    def leg(prec):
        c = copy.deepcopy(ctrl)
        c.precision = prec
        k = S.UnsCase(mesh, c, device=local)
        ier, _ = k.pimple_run(args.warmup, logcap=args.warmup)
        assert ier == 0, f"warm-up ier={ier}"
        rank_barrier(world)
        with ClockSampler(local) as clk:
            t0 = time.perf_counter()
            ier, log = k.pimple_run(args.steps, logcap=args.steps)
            wall = time.perf_counter() - t0
        rank_barrier(world)
        assert ier == 0 and len(log) == args.steps, (ier, len(log))
        tm = k.timing()
        mx = max_over_ranks(tm["total_ms"], world)
        return k, log, tm, mx, clk, wall

    k64, log64, _, mx64, _, _ = leg(abi.PREC_FP64)
    f64 = k64.fields()
    k64.close()
    case, log, tm, mx, clk, wall = leg(abi.PREC_MIXED if mixed else abi.PREC_FP64)
    value = job_rate(args.steps, world, mx)
    f = case.fields()
    rel = {k: float(np.linalg.norm(f[k] - f64[k]) / np.linalg.norm(f64[k])) for k in ("u", "p", "flux")}
    # end to end through the public API: host fields in (page-locked), one time
    # step, fields out into page-locked arrays
    hbuf = pinned_fields(case)
    case.fields(out=hbuf)
    h2d = (3 * N + N + F) * 8
    d2h = (3 * N + N + F + 3 * N + 9 * N + N) * 8
    rank_barrier(world)
    e2e_steps = max(2, min(args.steps, 20))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        case.upload(u=hbuf["u"], p=hbuf["p"], flux=hbuf["flux"])
        ier, _ = case.pimple_run(1, logcap=1)
        case.fields(out=hbuf)
    e2e_t = max_over_ranks(time.perf_counter() - t0, world)
    out = {
        "metric": PIMPLE_METRIC, "value": value, "unit": "time_steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mx / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": value / (world * PIMPLE_PUBLISHED_STEPS_PER_S),
        "dtype": "f32-inner/f64-refinement" if mixed else "f64",
        "data": "synthetic (the reference's 80 x 80 x 1 cavity layout, generated)",
        "config": {"workload": "transient PIMPLE, 2-D lid-driven cavity Re 1000, 80x80x1 hex (6400 cells), dt 0.01, "
                               "2 outer x 2 pressure corrections, alpha_u 0.7, conv_blend 1, lin_tol 1e-8; "
                               + ("mixed form: FP32-inner/FP64-refinement BiCGStab-Jacobi and PCG with "
                                  "Chebyshev-Jacobi" if mixed else "FP64 form: ILU(0) momentum, IC(0) PPE"),
                   "cells": N, "faces": F, "parallelism": f"replicas x{world}",
                   "l2": "working set ~5 MB fits L2 (as the reference's own run)",
                   "published": "0.182 s/step (5.5 steps/s), CPU MPI np=4, cluster_cases/cavity_Re1000/README.md:118",
                   "linear_iterations_per_step_max": int(max(r["itl_max"] for r in log)),
                   "fp64_form": {"time_steps_per_s": job_rate(args.steps, world, mx64),
                                 "linear_iterations_per_step_max": int(max(r["itl_max"] for r in log64)),
                                 "solvers": "BiCGStab+ILU(0) momentum, PCG+IC(0) pressure (exact sweeps, parity form)"},
                   "rel_l2_vs_fp64": rel, "rel_l2_after_steps": args.warmup + args.steps,
                   "t_end": log[-1]["t_now"]},
        "roofline": None,
        "e2e": {"value": world * e2e_steps / e2e_t, "unit": "time_steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": tm["gpu_launches"],
        "clocks": clk.summary(),
        "wall_s": wall,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:  # the CPU baseline is an N = 1 figure
        from oracle import oracle as O
        oc = O.OracleCase(mesh, ctrl)
        k = 5
        t0 = time.perf_counter()
        ier, _ = oc.pimple_run(k)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": k / dt, "unit": "time_steps/s", "cores": 1, "kind": "port",
                               "sample": f"{k} PIMPLE steps of the same cavity from rest, {dt:.1f} s"}
    case.close()
    close_ranks(world)
    if rank == 0:
        if getattr(args, "tuning_set", None):
            out["config"]["tuning"] = args.tuning_set
        print(json.dumps(out), flush=True)


def batch_specs(ncases, seed=0):
    """Cube edges with cell counts log-uniform in [16^3, 64^3] and Re uniform in
    [100, 2000], seeded: the batched workload's 3-D lid-driven cavities."""
    rng = np.random.default_rng(seed)
    cells = np.exp(rng.uniform(np.log(4096), np.log(262144), ncases))
    edges = np.clip(np.round(np.cbrt(cells)).astype(int), 16, 64)
    res = rng.uniform(100.0, 2000.0, ncases)
    return [(int(e), float(r), int(seed * 100003 + k)) for k, (e, r) in enumerate(zip(edges, res))]


def _batch_mesh(spec):
    from mixsolver_b200 import cases
    e, re, sd = spec
    return cases.cavity3d(e, re=re, seed=sd, outer_max=100)


def run_batch(args):
    """Batched workload: N independent 3-D lid-driven cavities (jittered hex,
    n^3 cells log-uniform in [4,096, 262,144], Re uniform in [100, 2000]),
    mixed-precision SIMPLE, all advanced by one batch: one launch per assembly
    kernel, one persistent lane launch per Krylov phase, the iteration replayed
    from a CUDA graph, lane policy from the autotuner. A step is one outer
    iteration of every case; `value` counts case-iterations per second."""
    rank, world, local = dist_env()
    import copy
    import torch
    torch.cuda.set_device(local)
    from mixsolver_b200 import abi
    from mixsolver_b200 import solver as S
    init_ranks(world)
    # one global set of cases; with several ranks each takes a balanced share of
    # whole cases (every rank computes the same assignment, no exchange)
    from mixsolver_b200 import shard
    specs = batch_specs(args.cases, seed=0)
    specs = [specs[i] for i in shard.mine([e ** 3 for e, _, _ in specs], world, rank)]
    t0 = time.perf_counter()
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        meshes = pool.map(_batch_mesh, specs)
    t_mesh = time.perf_counter() - t0
    cells = np.array([m.ncells for m, _ in meshes])
    nnz = np.array([m.ncells + 2 * m.n_interior() for m, _ in meshes])

    def make(prec):
        objs = []
        for mesh, ctrl in meshes:
            c = copy.deepcopy(ctrl)
            c.precision = prec
            c.lin_max = args.lin_max
            c.mom_solver = abi.MOM_JACOBI
            c.ppe_precond = abi.PPE_IC0
            objs.append(S.UnsCase(mesh, c, device=local))
        return objs

    t0 = time.perf_counter()
    objs = make(abi.PREC_MIXED)
    t_create = time.perf_counter() - t0
    dev_bytes = sum(o.device_bytes() for o in objs)
    nprof = 2  # profiled iterations after the timed ones (phase times, lane balance)
    for o in objs:
        assert o.begin(0, args.warmup + args.steps + nprof) == 0
    policy = None if args.policy == "auto" else tuple(int(v) for v in args.policy.split("x"))
    B = S.CaseBatch(objs, policy=policy)
    B.step(args.warmup)
    rank_barrier(world)
    i0 = B.info()
    with ClockSampler(local) as clk:
        w0 = time.perf_counter()
        active = B.step(args.steps)
        wall = time.perf_counter() - w0
    rank_barrier(world)
    i1 = B.info()
    ms = max_over_ranks(i1["step_ms"] - i0["step_ms"], world)
    value = args.cases * args.steps / (ms / 1e3)   # all ranks' case-iterations over the slowest rank's time
    B.set_profiling(True)
    B.step(nprof)
    ip = B.info()
    fin = [o.finish(logcap=args.warmup + args.steps + nprof) for o in objs]
    assert all(e == 0 for e, _ in fin), [e for e, _ in fin]
    timed = slice(args.warmup, args.warmup + args.steps)
    its = np.array([[sum(r["lin_it"][:3]), r["lin_it"][3]] for _, log in fin for r in log[timed]])
    # algorithmic bytes of the timed Krylov phases (same model as the single-case line)
    kbytes = 0.0
    for (_, log), n, z in zip(fin, cells, nnz):
        for r in log[timed]:
            kbytes += sum(krylov_bytes(int(n), int(z), r["lin_it"][c], "bicg", True) for c in range(3))
            kbytes += krylov_bytes(int(n), int(z), r["lin_it"][3], "pcg", True)
    # e2e through the public API: host fields of every case in (page-locked), one
    # batched iteration, every case's fields out into page-locked arrays
    hf = [pinned_fields(o) for o in objs]
    for o, f in zip(objs, hf):
        o.fields(out=f)
    for o in objs:
        o.begin(0, 10 ** 6)
    B2 = S.CaseBatch(objs, policy=(i1["split_rows"], i1["wide_lanes"]))
    B2.step(1)
    e2e_steps = 3
    w0 = time.perf_counter()
    for _ in range(e2e_steps):
        for o, f in zip(objs, hf):
            o.upload(u=f["u"], p=f["p"], flux=f["flux"])
        B2.step(1)
        for o, f in zip(objs, hf):
            o.fields(out=f)
    e2e_t = max_over_ranks(time.perf_counter() - w0, world)
    F = np.array([m.nfaces for m, _ in meshes])
    h2d = int(np.sum((5 * cells + F) * 8))
    d2h = int(np.sum((18 * cells + F) * 8))
    B2.close()
    B.close()
    for o in objs:
        o.close()
    # FP64 form over the first iterations of the same cases (comparison leg)
    objs64 = make(abi.PREC_FP64)
    for o in objs64:
        assert o.begin(0, args.fp64_iters) == 0
    B64 = S.CaseBatch(objs64)
    B64.step(args.fp64_iters)
    ms64 = B64.info()["step_ms"]
    value64 = args.cases * args.fp64_iters / (ms64 / 1e3)
    B64.close()
    for o in objs64:
        o.close()
    peak, peak_source = hbm_peak()
    achieved = kbytes / (ms / 1e3) / 1e9
    out = {
        "metric": "batched SIMPLE case-iterations/s (mixed precision, one persistent kernel per Krylov phase)",
        "value": value, "unit": "case_iters/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32-inner/f64-refinement", "data": "synthetic (seeded jittered hex cavities)",
        "config": {"workload": f"{args.cases} 3-D lid-driven cavities, n^3 hex cells log-uniform in "
                               "[4096, 262144], Re uniform in [100, 2000], mixed SIMPLE, lin_tol 1e-8",
                   "cells_total": int(cells.sum()), "cells_min": int(cells.min()), "cells_max": int(cells.max()),
                   "device_gb": dev_bytes / 1e9, "mesh_gen_s": t_mesh, "case_create_s": t_create,
                   "policy": {"split_rows": i1["split_rows"], "wide_lanes": i1["wide_lanes"],
                              "autotuned": i1["autotuned"], "tune_ms": i1["tune_ms"]},
                   "graph": i1["graph"], "launches_per_iter": i1["launches_per_iter"],
                   "pressure_lanes": i1["lanes"], "pressure_blocks": i1["blocks"],
                   "profile_per_iter_ms": {
                       "momentum": [v / nprof for v in ip["phase_ms"][:3]],
                       "pressure": [v / nprof for v in ip["phase_ms"][3:] if v > 0],
                       "assembly": ip["asm_ms"] / nprof,
                       "pressure_lane_busiest": ip["lane_max_ms"] / nprof,
                       "pressure_lane_mean": ip["lane_mean_ms"] / nprof},
                   "cell_iters_per_s": float(cells.sum()) * args.steps / (ms / 1e3),
                   "krylov_iterations_per_case_iter": {"momentum": float(its[:, 0].mean()),
                                                       "pressure": float(its[:, 1].mean())},
                   "fp64_form": {"case_iters_per_s": value64, "iters": args.fp64_iters,
                                 "solvers": "BiCGStab+Jacobi momentum, PCG+IC(0) pressure, cases one by one"},
                   "speedup_vs_fp64": value / value64,
                   "l2": "working set ~GBs > 126 MB L2"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "whole batched iteration (Krylov bytes / step time)",
                     "peak_source": peak_source},
        "e2e": {"value": world * args.cases * e2e_steps / e2e_t, "unit": "case_iters/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": i1["gpu_launches"] - i0["gpu_launches"],
        "clocks": clk.summary(), "wall_s": wall, "active_after": active,
    }
    close_ranks(world)
    if rank == 0:
        if getattr(args, "tuning_set", None):
            out["config"]["tuning"] = args.tuning_set
        print(json.dumps(out), flush=True)


# mesh pool of the served workload: jittered-hex cavities (SIMPLE) and
# hex-split-tet boxes (PISO) with cell counts spread over [1e4, 2e6]
SERVE_HEX_EDGES = (22, 30, 41, 56, 77, 105, 126)
SERVE_TET_EDGES = (12, 17, 24, 34, 48, 69)


def _serve_mesh(spec):
    from mixsolver_b200 import meshgen
    kind, e = spec
    if kind == "hex":
        return meshgen.sort_faces(meshgen.box_hex(e, e, e, jitter=0.10, seed=e, zones=(5, 5, 5, 5, 5, 5)))
    return meshgen.box_tet(e, wall_zone=4)


def serve_requests(duration, rate, pool, prec, seed=0):
    """Seeded Poisson arrivals: 70 % SIMPLE steady solves (50 outer
    iterations, lid-driven jittered-hex cavity), 30 % PISO batches (10 steps,
    dt = 1e-3, 2 correctors, Taylor-Green start in a walled hex-split-tet box);
    cells log-uniform in [1e4, 2e6] (nearest pool mesh), Re uniform in [50, 2000]."""
    import copy
    from mixsolver_b200 import abi, serve
    from mixsolver_b200.abi import BC_WALL, MOM_JACOBI, PPE_IC0, BcSpec, Ctrl
    rng = np.random.default_rng(seed)
    reqs, t, k = [], 0.0, 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        piso = rng.random() < 0.3
        cells = float(np.exp(rng.uniform(np.log(1e4), np.log(2e6))))
        re = float(rng.uniform(50.0, 2000.0))
        kind = "tet" if piso else "hex"
        mesh, xc = min(pool[kind], key=lambda mx: abs(np.log(mx[0].ncells / cells)))
        if piso:
            ctrl = Ctrl(rho=1.0, mu=1.0 / re, outer_max=1, lin_tol=1e-8, lin_max=1000, ppe_precond=PPE_IC0,
                        mom_solver=MOM_JACOBI, transient=True, time_scheme=1, dt=1e-3, n_time_max=10, n_correct=2,
                        bcs=[BcSpec(zone=4, btype=BC_WALL)])
            from mixsolver_b200 import meshgen
            u0 = meshgen.taylor_green(xc, seed=k)
        else:
            ctrl = Ctrl(rho=1.0, mu=1.0 / re, alpha_u=0.7, alpha_p=0.3, outer_max=50, outer_tol=0.0, lin_tol=1e-8,
                        lin_max=1000, ppe_precond=PPE_IC0, mom_solver=MOM_JACOBI,
                        bcs=[BcSpec(zone=5, btype=BC_WALL, lid=(2, 1.0, (1.0, 0.0, 0.0)))])
            u0 = None
        ctrl.precision = prec
        reqs.append(serve.Request(rid=k, arrival=t, mode=1 if piso else 0, mesh=mesh, ctrl=ctrl,
                                  nsteps=10 if piso else 50, u0=u0))
        k += 1
    return reqs


def run_serve(args):
    """Served workload: requests arrive as a Poisson stream while others are on
    the GPU; cases stay resident in HBM, are admitted against a memory budget,
    and are stepped by continuous batching. `value` is completed requests per
    second; p50 / p99 latency (arrival to result) beside it, for the mixed form
    and for the plain FP64 form (a shorter stream)."""
    rank, world, local = dist_env()
    import multiprocessing as mp
    import torch
    specs = [("hex", e) for e in SERVE_HEX_EDGES] + [("tet", e) for e in SERVE_TET_EDGES]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(min(13, os.cpu_count() or 1)) as pool:
        meshes = pool.map(_serve_mesh, specs)
    torch.cuda.set_device(local)
    from mixsolver_b200 import abi, serve
    from mixsolver_b200 import solver as S
    mpool = {"hex": [], "tet": []}
    for (kind, _), m in zip(specs, meshes):
        xc = S.compute_geometry(m)["xc"] if kind == "tet" else None
        mpool[kind].append((m, xc))
    t_pool = time.perf_counter() - t0
    budget = args.budget_gb * 1e9
    # warm-up: W requests on the smallest pool meshes, all arriving at once,
    # served before the timed streams (streams, modules, batch paths)
    small = {k: [min(v, key=lambda mx: mx[0].ncells)] for k, v in mpool.items()}
    wreqs = serve_requests(60.0, args.rate, small, abi.PREC_MIXED, seed=rank + 1000)[:max(args.warmup, 0)]
    for r in wreqs:
        r.arrival = 0.0
    if wreqs:
        wsrv = serve.Server(serve.GpuBackend(device=local, policy=(32768, 4)), budget_bytes=budget,
                            active_cells=args.active_cells, tick_iters=5)
        wout = wsrv.run(wreqs)
        assert all(r.error is None and r.ier == 0 for r in wout), [(r.rid, r.ier, r.error) for r in wout]
    legs = {}
    for name, prec, dur in (("mixed", abi.PREC_MIXED, args.duration), ("fp64", abi.PREC_FP64, args.fp64_duration)):
        reqs = serve_requests(dur, args.rate, mpool, prec, seed=0)
        if world > 1:  # every rank replays the same stream and keeps the requests routed to it
            from mixsolver_b200 import shard
            router = shard.Router(world)
            reqs = [r for r in reqs if router.route(r.arrival, r.cells * r.nsteps * 1e-7) == rank]
        srv = serve.Server(serve.GpuBackend(device=local, policy=(32768, 4)), budget_bytes=budget,
                           active_cells=args.active_cells, tick_iters=5)
        with ClockSampler(local) as clk:
            w0 = time.perf_counter()
            out = srv.run(reqs)
            wall = time.perf_counter() - w0
        sm = serve.summary(out, wall)
        sm.update({"wall_s": wall, "arrival_window_s": dur, "ticks": srv.ticks, "batches_built": srv.batches_built,
                   "peak_resident_gb": srv.peak_resident_bytes / 1e9,
                   "cells_min": min(r.cells for r in out), "cells_max": max(r.cells for r in out),
                   "simple": sum(1 for r in out if r.mode == 0), "piso": sum(1 for r in out if r.mode == 1),
                   "failed": [(r.rid, r.ier, r.error) for r in out if r.ier != 0 or r.error][:5],
                   "loop_s": {"build": srv.t_build, "step": srv.t_step, "finish": srv.t_finish},
                   "gpu_launches": srv.gpu_launches,
                   "per_request": [(r.rid, r.mode, r.cells, round(r.arrival, 3), round(r.admitted, 3),
                                    round(r.create_s, 3), round(r.finished, 3), r.nrec) for r in out][:60],
                   "clocks": clk.summary()})
        if world > 1:  # whole job: every rank's requests, over the slowest rank's wall time
            import torch.distributed as dist
            allr = [None] * world
            dist.all_gather_object(allr, [(r.finished - r.arrival) for r in out if r.error is None and r.ier == 0])
            lat = [x for part in allr for x in part]
            wmax = max_over_ranks(wall, world)
            sm["throughput_req_s"] = len(lat) / wmax
            sm["completed"] = len(lat)
            sm["p50_s"] = float(np.percentile(lat, 50)) if lat else None
            sm["p99_s"] = float(np.percentile(lat, 99)) if lat else None
            sm["wall_s"] = wmax
        legs[name] = sm
    mx = legs["mixed"]
    out = {
        "metric": "served SIMPLE/PISO requests: throughput with p50/p99 latency (mixed precision)",
        "value": mx["throughput_req_s"], "unit": "req/s", "n_gpus": world, "steps": mx["requests"],
        "warmup": len(wreqs),
        "ms_per_step": 1e3 * mx["wall_s"] / max(mx["completed"], 1), "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32-inner/f64-refinement",
        "data": "synthetic (seeded Poisson arrivals, jittered-hex and hex-split-tet meshes)",
        "config": {"workload": f"Poisson arrivals at {args.rate}/s: 70% SIMPLE (50 outer iterations, lid-driven "
                               "jittered-hex cavity), 30% PISO (10 steps, dt 1e-3, Taylor-Green hex-split-tet box); "
                               "cells log-uniform in [1e4, 2e6] (pool of 13 meshes), Re uniform in [50, 2000]",
                   "budget_gb": args.budget_gb, "active_cells": args.active_cells, "mesh_pool_s": t_pool, "latency_s": {"p50": mx["p50_s"], "p99": mx["p99_s"]},
                   "mixed": mx, "fp64": legs["fp64"],
                   "note": (f"arrivals over {args.duration:g} s, the last request answered after {mx['wall_s']:.1f} s: "
                            + ("the arrival rate exceeds the GPU's service rate, so latency is mostly queueing"
                               if mx["wall_s"] > 1.5 * args.duration + 30.0 else
                               "the GPU keeps up with the arrivals, so latency is mostly service time"))},
        "roofline": None,
        "e2e": {"value": mx["throughput_req_s"], "unit": "req/s", "h2d_bytes_per_step": None,
                "d2h_bytes_per_step": None},
        "gpu_launches": mx["gpu_launches"],
        "clocks": mx["clocks"],
    }
    if rank == 0:
        if getattr(args, "tuning_set", None):
            out["config"]["tuning"] = args.tuning_set
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    a = parse()
    if a.impl != "reference":
        a.tuning_set = apply_tuning(a)
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "batch":
        run_batch(a)
    elif a.workload == "serve":
        run_serve(a)
    elif a.workload == "piso":
        run_piso(a)
    elif a.workload == "pimple":
        run_pimple(a)
    else:
        run_ours(a)
