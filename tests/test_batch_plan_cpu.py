"""Lane planner of the batched Krylov launches (host logic, no GPU).

The mixed-precision solves give the same result on any number of blocks, so
the planner only balances: systems above the row threshold (or too big for
one block) go to the wide lanes, the others to single-block lanes; the lanes
fit the co-resident capacity, a wide lane is wide enough for the biggest
system, the blocks are split by the classes' share of the work, and the plan
depends only on its inputs."""
import numpy as np
import pytest

from mixsolver_b200 import abi
from mixsolver_b200 import solver as S

BLOCK_MAX_ROWS = 32768
SUPER = 256


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


def least_width(n):
    return max(1, -(-(-(-n // SUPER)) // (BLOCK_MAX_ROWS // SUPER)))


@pytest.mark.parametrize("split,wide,cap", [(32768, 8, 296), (8192, 2, 296), (16384, 16, 148), (32768, 4, 40)])
def test_plan_invariants(split, wide, cap):
    rows = sizes()
    passes = 17.0 * np.maximum(5.0, np.cbrt(rows))
    cls, widths = S.batch_plan(rows, split, wide, cap, passes=passes)
    big = (rows > split) | np.array([least_width(int(n)) > 1 for n in rows])
    assert np.all(cls[~big] == cls.max()) and np.all(cls[big] < cls.max()) if big.any() and (~big).any() else True
    assert widths.sum() <= cap and np.all(widths >= 1)
    nwide = int(np.sum(widths > 1)) if big.any() else 0
    assert nwide <= wide
    if big.any():
        need = max(least_width(int(n)) for n in rows[big])
        assert widths[:max(nwide, 1)].min() >= need
        work = passes * rows
        share = widths[:max(nwide, 1)].sum() / cap
        assert abs(share - work[big].sum() / work.sum()) < 0.05 + need / cap


def test_plan_is_deterministic():
    rows = sizes(seed=3)
    a = S.batch_plan(rows, 32768, 8, 296)
    b = S.batch_plan(rows, 32768, 8, 296)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_only_small_systems_get_one_lane_each_up_to_capacity():
    rows = np.full(10, 5000, np.int32)
    cls, widths = S.batch_plan(rows, 32768, 8, 296)
    assert np.all(cls == 0) and len(widths) == 10 and np.all(widths == 1)


def test_only_big_systems_share_the_whole_capacity():
    rows = np.array([300000, 70000, 100000], np.int32)
    cls, widths = S.batch_plan(rows, 32768, 8, 296)
    assert len(widths) == 3 and widths.sum() == 296
    # one class per big system, widest lane first, its system on it
    assert sorted(cls) == [0, 1, 2] and cls[0] == 0 and list(widths) == sorted(widths, reverse=True)


def test_plan_rejects_bad_arguments():
    with pytest.raises(RuntimeError):
        S.batch_plan(np.array([10], np.int32), 32768, 0, 100)
    with pytest.raises(RuntimeError):
        S.batch_plan(np.array([10], np.int32), 65536, 4, 100)


def test_few_big_systems_get_lanes_in_proportion_to_their_work():
    rows = np.array([2_000_000, 500_000, 100_000], np.int32)
    passes = np.array([100.0, 100.0, 100.0])
    cls, widths = S.batch_plan(rows, 32768, 4, 296, passes=passes)
    assert list(cls) == [0, 1, 2] and len(widths) == 3 and widths.sum() == 296
    share = widths / widths.sum()
    assert np.allclose(share, rows / rows.sum(), atol=0.03)
    for i, n in enumerate(rows):  # system i's lane is lane cls[i]: wide enough for it
        assert widths[cls[i]] >= least_width(int(n))


def test_narrow_lanes_never_take_a_system_wider_than_planned():
    """A few huge systems and small ones: each big system has a class of its
    own whose lane is wide enough for it, big classes are numbered widest lane
    first (a lane that takes from a later class meets only systems planned for
    narrower lanes), and the small systems form the last class."""
    rows = np.array([2_000_000, 1_157_625, 1_157_625, 456_533, 27_000, 10_000], np.int32)
    cls, widths = S.batch_plan(rows, 32768, 4, 280)
    big = rows > 32768
    assert sorted(cls[big]) == list(range(int(big.sum())))
    assert np.all(cls[~big] == big.sum())
    for i in np.nonzero(big)[0]:
        assert widths[cls[i]] >= least_width(int(rows[i]))
    nbig = int(big.sum())
    assert list(widths[:nbig]) == sorted(widths[:nbig], reverse=True)
    assert widths.sum() <= 280
