"""Lane planner of the batched Krylov launches (host logic, no GPU).

The mixed-precision solves give the same result on any number of blocks, so
the planner only balances: each system gets a lane width between 1 and its
super-chunk count (capped by the capacity), the lanes fit the co-resident
capacity, no lane's modelled load exceeds the makespan it reports, that
makespan is no shorter than the longest system on its widest lane, and the
plan depends only on its inputs."""
import numpy as np
import pytest

from mixsolver_b200 import abi
from mixsolver_b200 import solver as S


@pytest.fixture(scope="module", autouse=True)
def lib():
    from mixsolver_b200 import build
    build.build()
    return abi.load_library()


def sizes(k=256, seed=0):
    """Cubes whose cell counts are log-uniform in [16^3, 64^3]."""
    rng = np.random.default_rng(seed)
    cells = np.exp(rng.uniform(np.log(4096), np.log(262144), k))
    edge = np.clip(np.round(np.cbrt(cells)).astype(int), 16, 64)
    return (edge ** 3).astype(np.int32)


SUPER = 256  # rows of a super-chunk


def sys_time(n, p, w, bar_us, row_us):
    nsc = -(-n // SUPER)
    per = -(-nsc // w)
    rows = min(n, per * SUPER)
    return p * (rows * row_us + (bar_us if w > 1 else 0.05))


@pytest.mark.parametrize("bar_ns,row_ps,cap", [(1500, 6000, 296), (750, 4000, 296), (3000, 8000, 148),
                                               (1500, 6000, 40)])
def test_plan_invariants(bar_ns, row_ps, cap):
    rows = sizes()
    passes = 17.0 * np.maximum(5.0, np.cbrt(rows))
    w, lane, mk = S.batch_plan(rows, bar_ns, row_ps, cap, passes=passes)
    bar_us, row_us = bar_ns * 1e-3, row_ps * 1e-6
    nsc = -(-rows // SUPER)
    assert np.all(w >= 1) and np.all(w <= np.minimum(nsc, cap))
    widths = {}
    loads = {}
    for i, l in enumerate(lane):
        assert widths.setdefault(l, w[i]) == w[i]          # one width per lane
        loads[l] = loads.get(l, 0.0) + sys_time(int(rows[i]), passes[i], int(w[i]), bar_us, row_us)
    assert sum(widths.values()) <= cap
    assert max(loads.values()) <= mk * (1 + 1e-9)
    lower = max(sys_time(int(n), p, int(min(cap, -(-n // SUPER))), bar_us, row_us) for n, p in zip(rows, passes))
    assert mk >= lower * (1 - 1e-9)
    # within 2x of the work-conserving bound (all blocks busy, no barriers)
    work = sum(p * n * row_us for n, p in zip(rows, passes)) / cap
    assert mk <= 2.0 * max(work, lower) + 1e-9


def test_plan_is_deterministic():
    rows = sizes(seed=3)
    a = S.batch_plan(rows, 1500, 6000, 296)
    b = S.batch_plan(rows, 1500, 6000, 296)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]


def test_small_systems_share_a_lane_big_ones_spread():
    rows = np.array([1000, 5000, 300000, 70000], np.int32)
    w, lane, mk = S.batch_plan(rows, 1500, 6000, 296)
    assert w[0] == w[1] == 1 and lane[0] == lane[1]   # both fit one block within the makespan
    assert w[2] > w[3] > 1                            # the big systems spread over blocks
    assert len({lane[1], lane[2], lane[3]}) == 3


def test_plan_rejects_bad_arguments():
    with pytest.raises(RuntimeError):
        S.batch_plan(np.array([10], np.int32), 1500, 0, 100)
