"""The allocation-free PCG-Jacobi entry point (mgpu_cg_jacobi_noalloc).

It serves callers that may not allocate device memory (a host that owns all
device memory, CUDA Fortran device arrays): the caller passes device buffers,
the library works in one fixed internal array. Checked through the C-ABI
against the allocating entry point (mgpu_krylov_solve, cg_jacobi) with the
tolerances of the parity tests, on two calls in a row, so the second call also
shows the shared array is cleared; once on one block and once on several
blocks, where the array's grid-barrier counter and reduction partials are in
use; and on the early returns (b = 0, a row without a diagonal). This file is
collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from mixsolver_b200 import abi, cases
from mixsolver_b200 import solver as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _system(n=24, seed=0):
    """A pressure-correction matrix and rhs of the 2-D cavity (1-based CSR)."""
    mesh, ctrl = cases.cavity2d(n, outer_max=3)
    o = O.OracleCase(mesh, ctrl)
    o.simple_run()
    con = o.connectivity()
    aval, rhs, _ = o.stage(5, len(con["col_idx"]))
    rhs2 = rhs + 1e-3 * np.random.default_rng(seed).standard_normal(rhs.size)
    return con["row_ptr"], con["col_idx"], aval, rhs, rhs2


def _noalloc(lib, torch, rp, ci, val, b, x0, tol, maxit):
    dev = torch.device("cuda:0")
    d_rp = torch.tensor(rp - 1, dtype=torch.int32, device=dev)
    d_ci = torch.tensor(ci - 1, dtype=torch.int32, device=dev)
    d_val = torch.tensor(val, dtype=torch.float64, device=dev)
    d_b = torch.tensor(b, dtype=torch.float64, device=dev)
    d_x = torch.tensor(x0, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    it, ierr, res = C.c_int(), C.c_int(), C.c_double()
    rc = lib.mgpu_cg_jacobi_noalloc(len(rp) - 1, d_rp.data_ptr(), d_ci.data_ptr(), d_val.data_ptr(),
                                    d_b.data_ptr(), d_x.data_ptr(), tol, maxit, 0, None, C.byref(it),
                                    C.byref(res), C.byref(ierr))
    assert rc == 0, lib.mgpu_last_error()
    return d_x.cpu().numpy(), it.value, res.value, ierr.value


@pytest.fixture(params=["one_block", "multi_block"])
def layout(request):
    """One block, or the cooperative multi-block solve on 6 blocks (grid
    barrier and reduction partials inside the fixed array)."""
    if request.param == "multi_block":
        S.set_tuning("single_block_rows", 0)
        S.set_tuning("min_blocks", 6)
    yield request.param
    S.set_tuning("single_block_rows", 32768)
    S.set_tuning("min_blocks", 1)


def test_noalloc_matches_allocating_entry_point(gpu_lib, layout):
    torch = pytest.importorskip("torch")
    rp, ci, val, b1, b2 = _system()
    n = len(rp) - 1
    for b in (b1, b2):      # two calls in a row on the shared scratch array
        x0 = np.zeros(n)
        xa, ita, resa, ierra = _noalloc(gpu_lib, torch, rp, ci, val, b, x0, 1e-10, 500)
        xr, itr, resr, ierrr = S.cg_jacobi(rp, ci, val, b, x0, 1e-10, 500)
        assert (ita, ierra) == (itr, ierrr) and ierra == 0
        assert abs(resa - resr) <= 1e-3 * resr
        assert np.linalg.norm(xa - xr) / np.linalg.norm(xr) < 1e-9


def test_noalloc_early_returns_match(gpu_lib):
    """b = 0 gives x = 0 at iteration 0; a row without a diagonal gives
    ierr = 2 with x left as it was (cg_jacobi's contract), as the allocating
    entry point returns them."""
    torch = pytest.importorskip("torch")
    rp, ci, val, _, _ = _system(8)
    n = len(rp) - 1
    x0 = np.full(n, 0.5)
    xa, ita, resa, ierra = _noalloc(gpu_lib, torch, rp, ci, val, np.zeros(n), x0, 1e-8, 50)
    xr, itr, resr, ierrr = S.cg_jacobi(rp, ci, val, np.zeros(n), x0, 1e-8, 50)
    assert (ita, ierra) == (itr, ierrr) == (0, 0)
    np.testing.assert_array_equal(xa, xr)
    assert np.all(xa == 0.0)
    rp2 = np.array([1, 2, 3], np.int32)
    ci2 = np.array([2, 1], np.int32)        # no diagonal in either row
    v2 = np.array([1.0, 1.0])
    b2 = np.array([1.0, 1.0])
    x2 = np.array([0.25, -0.5])
    xa, ita, _, ierra = _noalloc(gpu_lib, torch, rp2, ci2, v2, b2, x2, 1e-8, 10)
    xr, itr, _, ierrr = S.cg_jacobi(rp2, ci2, v2, b2, x2, 1e-8, 10)
    assert (ita, ierra) == (itr, ierrr) and ierra == 2
    np.testing.assert_array_equal(xa, xr)


def test_noalloc_rejects_oversize(gpu_lib):
    n = abi.NOALLOC_MAX_ROWS + 1
    it, ierr, res = C.c_int(), C.c_int(), C.c_double()
    dummy = C.c_void_p(1)
    rc = gpu_lib.mgpu_cg_jacobi_noalloc(n, dummy, dummy, dummy, dummy, dummy, 1e-8, 10, 0, None,
                                        C.byref(it), C.byref(res), C.byref(ierr))
    assert rc == abi_status_arg()
    assert b"exceeds the fixed scratch limit" in gpu_lib.mgpu_last_error()


def abi_status_arg():
    return -1
