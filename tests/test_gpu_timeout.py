"""Failure detection on the device: a bounded grid-barrier wait that runs out.

Every spin-wait of the persistent Krylov kernels is bounded. When one runs out
the block flags DevStatus.timeout and returns; the other blocks see the flag at
their next poll and return too, and the host reports MGPU_E_TIMEOUT (-5). The
test lowers the poll limit to one poll (tuning key spin_limit), so any block of
a multi-block solve that has to wait gives up at once: no kernel hangs, nothing
faults, and the context stays usable. With the default limit restored the same
case must solve exactly as the oracle does.
"""
import numpy as np
import pytest

from mixsolver_b200 import abi, cases
from mixsolver_b200 import solver as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib(gpu_lib):
    return gpu_lib


@pytest.fixture
def multiblock():
    S.set_tuning("single_block_rows", 0)
    S.set_tuning("min_blocks", 6)
    yield
    S.set_tuning("spin_limit", 0)
    S.set_tuning("single_block_rows", 32768)
    S.set_tuning("min_blocks", 1)


def rel_l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("prec", [abi.PREC_FP64, abi.PREC_MIXED])
def test_barrier_wait_runs_out_then_case_recovers(prec, multiblock):
    # 3,456 cells: the multi-block launches hold 6 (FP64) and 7 (mixed) blocks,
    # so some block always has to wait at some barrier of the run
    mesh, ctrl = cases.channel3d(24, 12, 12, seed=3, outer_max=4, order_fn=S.rcm_order)
    ctrl.precision = prec
    ctrl.lin_max = 2000
    S.set_tuning("spin_limit", 1)
    g = S.UnsCase(mesh, ctrl)
    with pytest.raises(RuntimeError, match=r"status -5"):
        g.simple_run()
    S.set_tuning("spin_limit", 0)
    # the same case object runs again from rest with the default limit
    n = mesh.ncells
    g.upload(u=np.zeros((n, 3)), p=np.zeros(n), flux=np.zeros(mesh.nfaces))
    ier, log = g.simple_run()
    assert ier == 0 and len(log) == 4
    o = O.OracleCase(mesh, ctrl)
    ier_o, log_o = o.simple_run()
    assert ier_o == 0
    fg, fo = g.fields(), o.fields()
    tol = 1e-9 if prec == abi.PREC_FP64 else 1e-6
    for k in ("u", "p", "flux"):
        assert rel_l2(fg[k], fo[k]) < tol, k
    if prec == abi.PREC_FP64:
        assert [r["lin_it"] for r in log] == [r["lin_it"] for r in log_o]
