"""The mixed-precision form (FP32 inner Krylov inside FP64 refinement).

It uses Jacobi-preconditioned inner solves, so its iteration counts are not
the reference's; it must converge every system to the same tolerance on the
true FP64 residual and stay close to the FP64 parity form run over the same
outer iterations."""
import copy

import numpy as np
import pytest

from mixsolver_b200 import abi, cases, meshgen
from mixsolver_b200 import solver as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib(gpu_lib):
    return gpu_lib


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _pair(mesh, ctrl, steps, piso=False, u0=None):
    out = []
    for prec in (abi.PREC_FP64, abi.PREC_MIXED):
        c = copy.deepcopy(ctrl)
        c.precision = prec
        g = S.UnsCase(mesh, c)
        if u0 is not None:
            g.upload(u=u0)
        ier, log = g.piso_run(steps) if piso else g.simple_run(steps)
        assert ier == 0
        out.append((log, g.fields()))
    return out


@pytest.mark.parametrize("which", ["cavity", "channel"])
def test_mixed_simple_close_to_fp64(which):
    if which == "cavity":
        mesh, ctrl = cases.cavity2d(24, outer_max=30)
    else:
        mesh, ctrl = cases.channel3d(16, 8, 8, seed=4, outer_max=15, order_fn=S.rcm_order)
    ctrl.lin_max = 2000
    (l64, f64), (lmx, fmx) = _pair(mesh, ctrl, ctrl.outer_max)
    for r in lmx:
        assert all(e == 0 for e in r["lin_ierr"][:4]), r["lin_ierr"]
        assert all(x <= ctrl.lin_tol for x in r["lin_res"][:4])
    for k in ("u", "p", "flux"):
        assert rel(fmx[k], f64[k]) < 1e-6, (k, rel(fmx[k], f64[k]))


def test_mixed_multiblock_close_to_fp64():
    S.set_tuning("single_block_rows", 0)
    S.set_tuning("min_blocks", 6)
    try:
        mesh, ctrl = cases.channel3d(16, 8, 8, seed=5, outer_max=10, order_fn=S.rcm_order)
        ctrl.lin_max = 2000
        (l64, f64), (lmx, fmx) = _pair(mesh, ctrl, 10)
    finally:
        S.set_tuning("single_block_rows", 32768)
        S.set_tuning("min_blocks", 1)
    for k in ("u", "p", "flux"):
        assert rel(fmx[k], f64[k]) < 1e-6, (k, rel(fmx[k], f64[k]))


def test_mixed_piso_close_to_fp64():
    mesh, ctrl = cases.tet_box(4, dt=1e-3, steps=5)
    ctrl.lin_max = 2000
    u0 = meshgen.taylor_green(O.OracleCase(mesh, ctrl).geometry()["xc"], seed=3)
    (l64, f64), (lmx, fmx) = _pair(mesh, ctrl, 5, piso=True, u0=u0)
    for k in ("u", "p", "flux"):
        assert rel(fmx[k], f64[k]) < 1e-6, (k, rel(fmx[k], f64[k]))
