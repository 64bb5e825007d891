"""Whole-case sharding over ranks (mixsolver_b200.shard): two gloo ranks on the
CPU each compute their own share with no exchange of case lists; gathered,
the shares cover every case exactly once and their loads balance."""
import multiprocessing as mp
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from mixsolver_b200 import shard  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist
    from mixsolver_b200 import shard as sh
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    rng = np.random.default_rng(0)                     # the same inputs on every rank
    work = np.exp(rng.uniform(np.log(4096), np.log(262144), 256))
    mine = sh.mine(work, world, rank)
    # requests routed online: every rank replays the same stream
    r = sh.Router(world)
    arrivals = np.cumsum(rng.exponential(1 / 50.0, 200))
    service = rng.uniform(0.01, 0.2, 200)
    routed = [i for i, (a, s) in enumerate(zip(arrivals, service)) if r.route(a, s) == rank]
    got = [None] * world
    dist.all_gather_object(got, (mine, routed))
    dist.destroy_process_group()
    q.put((rank, got, float(work[mine].sum()), float(work.max())))


def test_two_gloo_ranks_shard_cases_without_exchange():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, got0, load0, wmax), (_, got1, load1, _) = out
    assert got0 == got1                                  # both ranks saw the same gather
    cases = sorted(got0[0][0] + got0[1][0])
    assert cases == list(range(256))                     # every case exactly once
    assert abs(load0 - load1) <= wmax                    # LPT bound
    reqs = sorted(got0[0][1] + got0[1][1])
    assert reqs == list(range(200))
    assert min(len(got0[0][1]), len(got0[1][1])) > 50     # both ranks serve


def test_assign_is_deterministic_and_balanced():
    w = [5, 3, 3, 2, 2, 2, 1]
    a = shard.assign(w, 3)
    assert a == shard.assign(list(w), 3)
    loads = [sum(x for x, r in zip(w, a) if r == k) for k in range(3)]
    assert sum(loads) == 18 and max(loads) - min(loads) <= max(w)
    assert a == [0, 1, 2, 1, 2, 0, 1]                     # largest first, least loaded, lower rank on ties
    assert shard.mine(w, 1, 0) == list(range(7))
