"""Serving loop logic (admission against the memory budget, active-set
selection, continuous batching) on a simulated backend: no GPU."""
import math
import threading

import numpy as np
import pytest

from mixsolver_b200 import serve


class _Mesh:
    def __init__(self, n):
        self.ncells = n


class FakeBackend:
    """Cases advance one iteration per stepped iteration until nsteps; device
    bytes are 1000 per cell. Records what the server asked for."""

    def __init__(self, bytes_per_cell=1000):
        self.bpc = bytes_per_cell
        self.lock = threading.Lock()
        self.live_bytes = 0
        self.peak_bytes = 0
        self.batches = []
        self.created = []

    def create(self, req):
        with self.lock:
            self.live_bytes += self.bpc * req.cells
            self.peak_bytes = max(self.peak_bytes, self.live_bytes)
            self.created.append(req.rid)
        return {"req": req, "done": 0, "open": True}, 0, self.bpc * req.cells

    def batch(self, handles):
        assert all(h["open"] for h in handles)
        self.batches.append([h["req"].rid for h in handles])
        return list(handles)

    def step(self, batch, iters):
        for h in batch:
            h["done"] = min(h["req"].nsteps, h["done"] + iters)

    def poll(self, batch):
        return np.array([int(h["done"] >= h["req"].nsteps) for h in batch])

    def finish(self, h, keep_fields):
        return 0, h["done"], None

    def release(self, h):
        h["open"] = False
        with self.lock:
            self.live_bytes -= self.bpc * h["req"].cells

    def close_batch(self, batch):
        pass


def _requests(k=40, seed=0):
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / 2000.0, k))
    return [serve.Request(rid=i, arrival=float(t[i]), mode=int(rng.random() < 0.3),
                          mesh=_Mesh(int(rng.integers(1000, 20000))), ctrl=None,
                          nsteps=int(rng.choice([10, 50]))) for i in range(k)]


def test_every_request_is_served_within_the_budget():
    be = FakeBackend()
    reqs = _requests()
    budget = 60_000_000  # 60 MB: a few cases at a time
    srv = serve.Server(be, budget_bytes=budget, active_cells=30000, tick_iters=5, bytes_per_cell=1000)
    out = srv.run(reqs)
    assert all(not math.isnan(r.finished) for r in out)
    assert all(r.nrec == r.nsteps for r in out)
    assert be.peak_bytes <= budget
    assert be.live_bytes == 0
    assert sorted(be.created) == sorted(r.rid for r in reqs)
    # admitted in arrival order
    adm = sorted(out, key=lambda r: r.admitted)
    assert [r.rid for r in adm] == [r.rid for r in sorted(out, key=lambda r: r.arrival)]
    for r in out:
        assert r.arrival <= r.admitted <= r.finished


def test_active_set_respects_the_cell_cap_and_prefers_short_work():
    be = FakeBackend()
    reqs = [serve.Request(rid=0, arrival=0.0, mode=0, mesh=_Mesh(10000), ctrl=None, nsteps=100),
            serve.Request(rid=1, arrival=0.0, mode=0, mesh=_Mesh(10000), ctrl=None, nsteps=10)]
    srv = serve.Server(be, budget_bytes=1e12, active_cells=10000, tick_iters=5, bytes_per_cell=1000)
    out = srv.run(reqs)
    for b in be.batches:
        assert len(b) == 1  # one case of 10000 cells fills the cap
    assert out[1].finished <= out[0].finished  # less remaining work goes first
    s = serve.summary(out, wall=max(r.finished for r in out))
    assert s["completed"] == 2 and s["ok"] == 2 and s["p50_s"] is not None


def test_a_case_bigger_than_the_budget_is_still_served_alone():
    be = FakeBackend()
    reqs = [serve.Request(rid=0, arrival=0.0, mode=0, mesh=_Mesh(5000), ctrl=None, nsteps=5)]
    srv = serve.Server(be, budget_bytes=1000, tick_iters=5, bytes_per_cell=1000)
    out = srv.run(reqs)
    assert out[0].nrec == 5


def test_rejected_case_is_answered_with_its_error():
    class Failing(FakeBackend):
        def create(self, req):
            if req.rid == 1:
                raise RuntimeError("mesh rejected")
            return super().create(req)

    be = Failing()
    reqs = [serve.Request(rid=i, arrival=0.0, mode=0, mesh=_Mesh(1000), ctrl=None, nsteps=5) for i in range(3)]
    out = serve.Server(be, budget_bytes=1e9, tick_iters=5).run(reqs)
    assert out[1].error == "mesh rejected" and not math.isnan(out[1].finished)
    assert out[0].nrec == 5 and out[2].nrec == 5


def test_launch_count_follows_the_ticks():
    """The server adds what the backend's own counter grew by over each tick
    (the library counts the kernels a batch runs, graph replays included)."""
    class Counting(FakeBackend):
        n = 0

        def step(self, batch, iters):
            super().step(batch, iters)
            self.n += 7 * iters

        def launches(self, batch):
            return self.n

    be = Counting()
    srv = serve.Server(be, budget_bytes=60_000_000, active_cells=30000, tick_iters=5, bytes_per_cell=1000)
    srv.run(_requests(k=12, seed=3))
    assert srv.ticks > 0 and srv.gpu_launches == 7 * 5 * srv.ticks
    plain = serve.Server(FakeBackend(), budget_bytes=60_000_000, active_cells=30000, tick_iters=5,
                         bytes_per_cell=1000)
    plain.run(_requests(k=4, seed=4))
    assert plain.gpu_launches == 0   # a backend without a count adds nothing
