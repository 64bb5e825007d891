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
