"""The mixed-precision form (FP32 inner Krylov inside FP64 refinement).

It uses Jacobi / Chebyshev-Jacobi preconditioned inner solves, so its
iteration counts are not the reference's; it must converge every system to the
same tolerance on the true FP64 residual, and its fields must stay within
1e-8 relative L2 of the converged FP64 answer of the same outer iterations
(the FP64 parity form solved to 1e-12)."""
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


TIGHT = 1e-12   # lin_tol of the FP64 reference the mixed form is held to
GATE = 1e-8     # relative L2 field error of the mixed form against it


def _run(mesh, ctrl, steps, prec, tol=None, piso=False, u0=None):
    c = copy.deepcopy(ctrl)
    c.precision = prec
    if tol is not None:
        c.lin_tol = tol
        c.lin_max = 4000
    g = S.UnsCase(mesh, c)
    if u0 is not None:
        g.upload(u=u0)
    ier, log = g.piso_run(steps) if piso else g.simple_run(steps)
    assert ier == 0
    return log, g.fields()


def _check(mesh, ctrl, steps, piso=False, u0=None):
    """The mixed form at the case's lin_tol against the FP64 parity form solved
    to TIGHT (the converged answer of the same outer iterations): every field
    within GATE. Against the FP64 form at the same lin_tol the difference is
    that form's own solve error (printed)."""
    lmx, fmx = _run(mesh, ctrl, steps, abi.PREC_MIXED, piso=piso, u0=u0)
    _, ftight = _run(mesh, ctrl, steps, abi.PREC_FP64, tol=TIGHT, piso=piso, u0=u0)
    _, f64 = _run(mesh, ctrl, steps, abi.PREC_FP64, piso=piso, u0=u0)
    for r in lmx:
        assert all(e == 0 for e in r["lin_ierr"][:4]), r["lin_ierr"]
        assert all(x <= ctrl.lin_tol for x in r["lin_res"][:4])
    errs = {k: rel(fmx[k], ftight[k]) for k in ("u", "p", "flux")}
    same_tol = {k: rel(f64[k], ftight[k]) for k in ("u", "p", "flux")}
    print("mixed vs tight FP64:", errs, "FP64 form at lin_tol vs tight:", same_tol)
    for k, v in errs.items():
        assert v < GATE, (k, v)


@pytest.mark.parametrize("which", ["cavity", "channel"])
def test_mixed_simple_meets_gate(which):
    if which == "cavity":
        mesh, ctrl = cases.cavity2d(24, outer_max=30)
    else:
        mesh, ctrl = cases.channel3d(16, 8, 8, seed=4, outer_max=15, order_fn=S.rcm_order)
    ctrl.lin_max = 2000
    _check(mesh, ctrl, ctrl.outer_max)


def test_mixed_multiblock_meets_gate():
    S.set_tuning("single_block_rows", 0)
    S.set_tuning("min_blocks", 6)
    try:
        mesh, ctrl = cases.channel3d(16, 8, 8, seed=5, outer_max=10, order_fn=S.rcm_order)
        ctrl.lin_max = 2000
        _check(mesh, ctrl, 10)
    finally:
        S.set_tuning("single_block_rows", 32768)
        S.set_tuning("min_blocks", 1)


def test_mixed_piso_meets_gate():
    mesh, ctrl = cases.tet_box(4, dt=1e-3, steps=5)
    ctrl.lin_max = 2000
    u0 = meshgen.taylor_green(O.OracleCase(mesh, ctrl).geometry()["xc"], seed=3)
    _check(mesh, ctrl, 5, piso=True, u0=u0)


def test_mixed_neighbour_sync_bit_identical():
    """The optional neighbour sync (tuning key neighbor_sync): a single-system
    pressure solve runs its Chebyshev passes on contiguous row ranges, each
    block waiting only for the blocks whose rows it reads. Every sum still runs
    over fixed row chunks, so the run is bit-identical to the same run with
    grid barriers (the default)."""
    mesh, ctrl = cases.channel3d(32, 16, 16, seed=6, outer_max=5, order_fn=S.rcm_order)
    ctrl.precision = abi.PREC_MIXED
    ctrl.lin_max = 2000
    out = []
    S.set_tuning("single_block_rows", 0)
    try:
        for ns in (1, 0):
            S.set_tuning("neighbor_sync", ns)
            g = S.UnsCase(mesh, ctrl)
            ier, log = g.simple_run()
            assert ier == 0
            out.append((log, g.fields()))
    finally:
        S.set_tuning("neighbor_sync", 0)
        S.set_tuning("single_block_rows", 32768)
    for a, b in zip(out[0][0], out[1][0]):
        assert a["lin_it"] == b["lin_it"] and a["lin_res"] == b["lin_res"]
    for k in ("u", "p", "flux"):
        np.testing.assert_array_equal(out[0][1][k], out[1][1][k])


def test_restarted_and_reliable_schemes_close():
    """The pressure PCG's two refinement schemes (restarted inner solves,
    reliable updates) converge the same systems to the same tolerance."""
    mesh, ctrl = cases.channel3d(16, 8, 8, seed=4, outer_max=8, order_fn=S.rcm_order)
    ctrl.precision = abi.PREC_MIXED
    ctrl.lin_max = 2000
    ctrl.lin_tol = 1e-11
    out = []
    try:
        for sch in (0, 1):
            S.set_tuning("mixed_scheme", sch)
            g = S.UnsCase(mesh, ctrl)
            ier, log = g.simple_run()
            assert ier == 0
            for r in log:
                assert all(e == 0 for e in r["lin_ierr"][:4]) and all(x <= 1e-11 for x in r["lin_res"][:4])
            out.append(g.fields())
    finally:
        S.set_tuning("mixed_scheme", 1)
    for k in ("u", "p", "flux"):
        assert rel(out[0][k], out[1][k]) < 1e-9, k


def test_fp64_poly_form_close_to_parity_form():
    """The mixed form's solvers in FP64 throughout (MGPU_PREC_FP64_POLY) against
    the FP64 parity form, both to lin_tol 1e-11: the same fields to 1e-8."""
    mesh, ctrl = cases.channel3d(16, 8, 8, seed=4, outer_max=10, order_fn=S.rcm_order)
    ctrl.lin_max = 2000
    ctrl.lin_tol = 1e-11
    fields = []
    for prec in (abi.PREC_FP64, abi.PREC_FP64_POLY):
        c = copy.deepcopy(ctrl)
        c.precision = prec
        g = S.UnsCase(mesh, c)
        ier, log = g.simple_run()
        assert ier == 0
        for r in log:
            assert all(e == 0 for e in r["lin_ierr"][:4]) and all(x <= 1e-11 for x in r["lin_res"][:4])
        fields.append(g.fields())
    for k in ("u", "p", "flux"):
        assert rel(fields[1][k], fields[0][k]) < 1e-8, (k, rel(fields[1][k], fields[0][k]))
