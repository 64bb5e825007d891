"""Serving: SIMPLE steady solves and PISO time-step batches of different sizes,
answered as they arrive, with continuous batching on one GPU.

The reference has no counterpart: it advances one case per process. Here a
request is a mesh plus a control (:class:`Request`), and :class:`Server` runs
two loops:

* an admission thread makes arriving cases resident in HBM (mesh, matrices,
  fields: ``mgpu_case_create`` + field upload + ``mgpu_case_begin``) in arrival
  order, whenever the device memory they need fits the budget beside the cases
  already resident; it works while the GPU steps the others (the native calls
  release the interpreter lock);
* the stepping loop advances the active set (the resident cases with the least
  remaining work, up to ``active_cells`` cells) ``tick_iters`` outer
  iterations / time steps at a time through one :class:`~mixsolver_b200.solver.CaseBatch`
  (one launch per assembly kernel, one persistent launch per Krylov phase);
  after each tick finished cases are read back and freed, and the active set
  is refilled, so requests join and leave between ticks.

With a fixed lane policy every case's result is bit-identical to the one it
gets when served alone (the mixed-precision solves do not depend on the lane
they run on; FP64 cases run the single-case solvers).

The server talks to the GPU through a backend (:class:`GpuBackend`); tests of
the scheduling logic use a simulated one.
"""
from __future__ import annotations

import dataclasses
import math
import threading
import time
from typing import Callable, List, Optional

import numpy as np


@dataclasses.dataclass
class Request:
    """One solve: ``mode`` 0 = SIMPLE steady (``nsteps`` outer iterations at
    most), 1 = PISO (``nsteps`` time steps); ``u0`` an optional initial
    velocity (ncells, 3); ``arrival`` seconds after the start of the run."""
    rid: int
    arrival: float
    mode: int
    mesh: object
    ctrl: object
    nsteps: int
    u0: Optional[np.ndarray] = None
    # filled in by the server
    admitted: float = math.nan
    create_s: float = math.nan  # seconds spent making the case resident
    finished: float = math.nan
    ier: int = -1
    nrec: int = 0
    device_bytes: int = 0
    fields: Optional[dict] = None
    error: Optional[str] = None

    @property
    def cells(self) -> int:
        return int(self.mesh.ncells)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class GpuBackend:
    """The C-ABI: a resident case per request, one CaseBatch per active set."""

    def __init__(self, device: int = 0, policy=(32768, 4), reserve_blocks: int = 16):
        from . import solver
        self.S = solver
        self.device = device
        self.policy = policy
        # leave block slots free during the batched Krylov launches so that the
        # set-up kernels of arriving cases run beside them
        solver.set_tuning("batch_reserve_blocks", int(reserve_blocks))
        # streams for the cases and batches to come, made before the GPU is busy
        solver.set_tuning("stream_pool", 64)

    def create(self, req: Request):
        c = self.S.UnsCase(req.mesh, req.ctrl, device=self.device)
        if req.u0 is not None:
            c.upload(u=req.u0)
        ier = c.begin(req.mode, req.nsteps)
        return c, ier, c.device_bytes()

    def batch(self, handles):
        return self.S.CaseBatch(handles, policy=self.policy)

    def step(self, batch, iters: int) -> None:
        batch.step(iters)

    def launches(self, batch) -> int:
        """Kernels the batch has run so far (the library's own count)."""
        return int(batch.info()["gpu_launches"])

    def poll(self, batch) -> np.ndarray:
        return batch.poll()

    def finish(self, h, keep_fields: bool):
        ier, log = h.finish(logcap=1 << 16)
        return ier, len(log), (h.fields() if keep_fields else None)

    def release(self, h) -> None:
        h.close()

    def close_batch(self, batch) -> None:
        batch.close()


class Server:
    """Continuous batching over resident cases (see the module docstring).

    budget_bytes: device memory the resident cases may hold together;
    active_cells: cells stepped together per tick (bounds the tick time);
    tick_iters:   outer iterations / time steps per tick;
    bytes_per_cell: device bytes a case is expected to need per cell before
                  it is created (refined from the cases created so far)."""

    def __init__(self, backend, budget_bytes: float, active_cells: int = 16_000_000, tick_iters: int = 4,
                 keep_fields: bool = False, clock: Callable[[], float] = time.perf_counter,
                 bytes_per_cell: float = 1500.0):
        self.be = backend
        self.budget = float(budget_bytes)
        self.active_cells = int(active_cells)
        self.tick_iters = int(tick_iters)
        self.keep_fields = keep_fields
        self.clock = clock
        self.bytes_per_cell = bytes_per_cell
        self.lock = threading.Condition()
        self.resident_bytes = 0
        self.peak_resident_bytes = 0
        self.ticks = 0
        self.batches_built = 0
        self.gpu_launches = 0  # batched-iteration launches stepped (backends that count them)
        self.case_iters = 0
        self.cell_iters = 0.0
        # wall seconds of the stepping loop: building batches, stepping,
        # reading back and releasing finished cases
        self.t_build = self.t_step = self.t_finish = 0.0

    # ---- admission -------------------------------------------------------
    def _estimate(self, req: Request) -> float:
        return self.bytes_per_cell * req.cells

    def _admit_loop(self, pending: List[Request], resident: list, t0: float, stop: threading.Event):
        seen_cells = seen_bytes = 0
        for req in pending:  # arrival order
            est = self._estimate(req)  # reserved while the case is created
            while not stop.is_set():
                now = self.clock() - t0
                if now < req.arrival:
                    time.sleep(min(0.002, req.arrival - now))
                    continue
                with self.lock:
                    est = self._estimate(req)
                    fits = self.resident_bytes + est <= self.budget or self.resident_bytes == 0
                    if fits:
                        self.resident_bytes += est
                    else:
                        self.lock.wait(0.01)
                if fits:
                    break
            if stop.is_set():
                return
            tc = self.clock()
            try:
                h, ier, nbytes = self.be.create(req)
            except Exception as e:  # a case the library rejects: answered with the error
                with self.lock:
                    self.resident_bytes -= est
                    req.error = str(e)
                    req.finished = self.clock() - t0
                    self.lock.notify_all()
                continue
            seen_cells += req.cells
            seen_bytes += nbytes
            with self.lock:
                self.resident_bytes += nbytes - est
                self.peak_resident_bytes = max(self.peak_resident_bytes, self.resident_bytes)
                self.bytes_per_cell = seen_bytes / max(seen_cells, 1)
                req.admitted = self.clock() - t0
                req.create_s = self.clock() - tc
                req.device_bytes = nbytes
                req.ier = ier
                resident.append([req, h, 0])  # request, handle, iterations stepped
                self.lock.notify_all()

    # ---- stepping --------------------------------------------------------
    def run(self, requests: List[Request]) -> List[Request]:
        """Serve every request; returns them with admission and completion
        times (seconds from the start), ier, records and (optionally) fields."""
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        resident: list = []
        stop = threading.Event()
        t0 = self.clock()
        adm = threading.Thread(target=self._admit_loop, args=(pending, resident, t0, stop), daemon=True)
        adm.start()
        done = 0
        batch, members = None, []
        try:
            while done < len(pending):
                with self.lock:
                    # requests rejected at creation count as done
                    done = sum(1 for r in pending if not math.isnan(r.finished))
                    if done >= len(pending):
                        break
                    cand = [e for e in resident if math.isnan(e[0].finished)]
                    if not cand:
                        self.lock.wait(0.005)
                        continue
                    # least remaining work first, up to active_cells
                    cand.sort(key=lambda e: ((e[0].nsteps - e[2]) * e[0].cells, e[0].arrival, e[0].rid))
                    active, cells = [], 0
                    for e in cand:
                        if active and cells + e[0].cells > self.active_cells:
                            continue
                        active.append(e)
                        cells += e[0].cells
                tb = self.clock()
                if [id(e[1]) for e in active] != [id(h) for h in members]:
                    if batch is not None:
                        self.be.close_batch(batch)
                    members = [e[1] for e in active]
                    batch = self.be.batch(members)
                    self.batches_built += 1
                ts = self.clock()
                count = getattr(self.be, "launches", None)
                n0 = int(count(batch)) if count is not None else 0
                self.be.step(batch, self.tick_iters)
                self.ticks += 1
                if count is not None:
                    self.gpu_launches += int(count(batch)) - n0
                flags = self.be.poll(batch)
                now = self.clock() - t0
                self.t_build += ts - tb
                self.t_step += now + t0 - ts
                finished = []
                for e, fl in zip(active, flags):
                    e[2] += self.tick_iters
                    if not fl:
                        continue
                    req, h = e[0], e[1]
                    ier, nrec, fields = self.be.finish(h, self.keep_fields)
                    if req.ier == 0:
                        req.ier = ier
                    req.nrec = nrec
                    req.fields = fields
                    self.case_iters += nrec
                    self.cell_iters += float(nrec) * req.cells
                    finished.append(e)
                tf = self.clock()
                if finished:
                    # the batch refers to the finished cases' arrays: drop it first
                    self.be.close_batch(batch)
                    batch, members = None, []
                    for e in finished:
                        self.be.release(e[1])
                        with self.lock:
                            e[0].finished = now
                            resident.remove(e)
                            self.resident_bytes -= e[0].device_bytes
                            self.lock.notify_all()
                self.t_finish += self.clock() - tf
        finally:
            stop.set()
            adm.join(timeout=30)
            if batch is not None:
                self.be.close_batch(batch)
            for e in resident:
                self.be.release(e[1])
        return pending


def summary(reqs: List[Request], wall: float) -> dict:
    """Latency percentiles (seconds) and throughput of a served run."""
    lat = np.array([r.latency for r in reqs if not math.isnan(r.finished)])
    ok = [r for r in reqs if r.error is None and r.ier == 0]
    pct = lambda q: float(np.percentile(lat, q)) if len(lat) else None
    return {"requests": len(reqs), "completed": int(len(lat)), "ok": len(ok),
            "p50_s": pct(50), "p99_s": pct(99), "mean_s": float(lat.mean()) if len(lat) else None,
            "throughput_req_s": len(lat) / wall if wall > 0 else None,
            "case_iters_per_s": sum(r.nrec for r in reqs) / wall if wall > 0 else None,
            "cell_iters_per_s": sum(r.nrec * r.cells for r in reqs) / wall if wall > 0 else None}
