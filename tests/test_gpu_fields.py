"""Host <-> device field copies through the C-ABI (mgpu_fields_upload /
mgpu_fields_download): the cell-major (Fortran u(3,ncells), gu(3,3,ncells))
layouts are transposed on the device, so a round trip and every read-back
layout are checked bit for bit here."""
import numpy as np
import pytest

from mixsolver_b200 import cases
from mixsolver_b200 import solver as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib(gpu_lib):
    return gpu_lib


def _case():
    mesh, ctrl = cases.cavity3d(12, outer_max=3)
    return S.UnsCase(mesh, ctrl)


def test_upload_download_round_trip():
    c = _case()
    rng = np.random.default_rng(3)
    u = rng.standard_normal((c.N, 3))
    p = rng.standard_normal(c.N)
    flux = rng.standard_normal(c.F)
    c.upload(u=u, p=p, flux=flux)
    f = c.fields()
    np.testing.assert_array_equal(f["u"], u)
    np.testing.assert_array_equal(f["p"], p)
    np.testing.assert_array_equal(f["flux"], flux)
    c.close()


def test_fields_out_matches_fields():
    c = _case()
    ier, _ = c.simple_run(3)
    assert ier == 0
    ref = c.fields()
    # gradients are not trivial after three iterations
    assert np.abs(ref["gu"]).max() > 0 and np.abs(ref["gp"]).max() > 0
    out = {k: np.full(v.shape, np.nan) for k, v in ref.items()}
    got = c.fields(out=out)
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    # the caller's gu array holds the C-ABI layout [cell, direction, component]
    np.testing.assert_array_equal(out["gu"], ref["gu"].transpose(0, 2, 1))
    # a subset reads back only what is asked for
    part = {"p": np.zeros(c.N)}
    got = c.fields(out=part)
    assert set(got) == {"p"}
    np.testing.assert_array_equal(part["p"], ref["p"])
    with pytest.raises(ValueError):
        c.fields(out={"u": np.zeros((c.N, 2))})
    c.close()


def _pinned(ref):
    import torch
    return {k: torch.empty(v.shape, dtype=torch.float64, pin_memory=True).numpy() for k, v in ref.items()}


@pytest.mark.parametrize("what", ["pinned", "pageable", "converges_early", "stops_at_check"])
def test_simple_run_fields_matches_run_then_download(what):
    """mgpu_simple_run_fields gives what mgpu_simple_run followed by
    mgpu_fields_download gives, bit for bit: with page-locked arrays (gp, gu
    and apc copied during the last iteration), pageable ones (all copied at
    the end), a run that converges before its last iteration (that iteration
    then changes nothing) and one that stops at the abort check after 64
    iterations, before its last one (everything copied at the end)."""
    mesh, ctrl = cases.cavity3d(12, outer_max=200)
    nsteps = 6
    if what == "converges_early":
        ctrl.outer_tol = 5e-2
        nsteps = 12
    elif what == "stops_at_check":
        ctrl.outer_tol = 5e-2
        nsteps = 100
    a, b = S.UnsCase(mesh, ctrl), S.UnsCase(mesh, ctrl)
    ier_a, log_a = a.simple_run(nsteps)
    ref = a.fields()
    out = _pinned(ref) if what != "pageable" else {k: np.empty(v.shape) for k, v in ref.items()}
    for k in out:
        out[k][...] = np.nan
    ier_b, log_b, got = b.simple_run_fields(nsteps, out=out)
    assert ier_a == ier_b == 0
    assert len(log_a) == len(log_b)
    if what in ("converges_early", "stops_at_check"):
        assert len(log_b) < nsteps
    for ra, rb in zip(log_a, log_b):
        assert ra["lin_it"] == rb["lin_it"] and ra["du_max"] == rb["du_max"]
    for k in ref:
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    # a second call on the same case (the copy stream and buffer reused)
    ier_a, _ = a.simple_run(2)
    ref2 = a.fields()
    ier_b, _, got2 = b.simple_run_fields(2, out=out)
    for k in ref2:
        np.testing.assert_array_equal(got2[k], ref2[k], err_msg=k)
    a.close()
    b.close()
