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


def _ppe(nx, ny, nz):
    """A pressure-correction system of the jittered channel after 3 oracle
    SIMPLE iterations (1-based CSR)."""
    mesh, ctrl = cases.channel3d(nx, ny, nz, seed=2, outer_max=3, order_fn=S.rcm_order)
    o = O.OracleCase(mesh, ctrl)
    o.simple_run()
    con = o.connectivity()
    aval, rhs, _ = o.stage(5, len(con["col_idx"]))
    return con["row_ptr"], con["col_idx"], aval, rhs


@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_FP64_POLY])
def test_pcg_poly_solve_on_a_csr_system(prec):
    """mgpu_pcg_poly_solve: converged on the FP64 residual (checked here with
    the oracle's csr_matvec), the same answer as cg_ic0 to the tolerance, and
    the same bits from one block and from a grid of blocks (layout-independent
    sums)."""
    rp, ci, aval, rhs = _ppe(24, 12, 12)
    x0 = np.zeros(len(rp) - 1)
    tol = 1e-10
    x1, it1, res1, ierr1 = S.pcg_poly(rp, ci, aval, rhs, x0, tol, 2000, prec)
    assert ierr1 == 0 and res1 <= tol and it1 > 0
    true = np.linalg.norm(rhs - O.csr_matvec(rp, ci, aval, x1)) / np.linalg.norm(rhs)
    assert true <= tol * (1 + 1e-6), true
    xr, _, _, ierr = S.cg_ic0(rp, ci, aval, rhs, x0, 1e-12, 2000)
    assert ierr == 0
    assert rel(x1, xr) < 1e-7, rel(x1, xr)
    S.set_tuning("single_block_rows", 0)
    try:
        x2, it2, res2, ierr2 = S.pcg_poly(rp, ci, aval, rhs, x0, tol, 2000, prec)
    finally:
        S.set_tuning("single_block_rows", 32768)
    assert (it2, ierr2) == (it1, ierr1) and res2 == res1
    np.testing.assert_array_equal(x2, x1)


def test_pcg_poly_solve_jacobi_and_iteration_cap():
    """Degree 1 is Jacobi PCG; a cap below the need returns ierr 1."""
    rp, ci, aval, rhs = _ppe(16, 8, 8)
    x0 = np.zeros(len(rp) - 1)
    x, it, res, ierr = S.pcg_poly(rp, ci, aval, rhs, x0, 1e-9, 5000, abi.PREC_MIXED, cheb_degree=1)
    assert ierr == 0 and res <= 1e-9
    _, it5, res5, ierr5 = S.pcg_poly(rp, ci, aval, rhs, x0, 1e-9, 5, abi.PREC_MIXED)
    assert ierr5 == 1 and res5 > 1e-9
