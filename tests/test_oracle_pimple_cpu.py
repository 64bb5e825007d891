"""The oracle's PIMPLE restatement (pimple_run_mpi at one rank) against its
PISO restatement: with alpha_u = 1 and one outer iteration per step the
momentum relaxation and apc = ap / alpha_u are identities, so both give the
same records and fields bit for bit; with relaxation and two outer iterations
the run differs and still converges every solve."""
import numpy as np

from mixsolver_b200 import cases, meshgen
from oracle import oracle as O


def _run(mesh, ctrl, u0, run):
    o = O.OracleCase(mesh, ctrl)
    o.upload(u=u0)
    ier, log = getattr(o, run)()
    return ier, log, o.fields()


def test_unrelaxed_single_outer_pimple_is_piso():
    mesh, ctrl = cases.tet_box(3, dt=1e-3, steps=3)
    ctrl.alpha_u = 1.0
    ctrl.n_outer_iter = 1
    u0 = meshgen.taylor_green(O.OracleCase(mesh, ctrl).geometry()["xc"], seed=5)
    a = _run(mesh, ctrl, u0, "piso_run")
    b = _run(mesh, ctrl, u0, "pimple_run")
    assert a[0] == b[0] == 0
    assert [r["lin_it"] for r in a[1]] == [r["lin_it"] for r in b[1]]
    assert [r["ressum"] for r in a[1]] == [r["ressum"] for r in b[1]]
    for key in ("u", "p", "flux"):
        np.testing.assert_array_equal(a[2][key], b[2][key])


def test_relaxed_outer_iterations_differ_and_converge():
    mesh, ctrl = cases.tet_box(3, dt=2e-3, steps=3)
    ctrl.alpha_u = 0.7
    ctrl.n_outer_iter = 2
    u0 = meshgen.taylor_green(O.OracleCase(mesh, ctrl).geometry()["xc"], seed=6)
    a = _run(mesh, ctrl, u0, "piso_run")
    b = _run(mesh, ctrl, u0, "pimple_run")
    assert a[0] == b[0] == 0
    assert all(max(r["lin_ierr"]) == 0 for r in b[1])
    assert not np.array_equal(a[2]["u"], b[2]["u"])
    # itl_max covers both outer iterations' solves
    assert all(r["itl_max"] >= max(r["lin_it"][:r["nsolve"]]) for r in b[1])


def test_pimple_error_codes():
    mesh, ctrl = cases.cavity2d(4)
    assert O.OracleCase(mesh, ctrl).pimple_run()[0] == 50
    ctrl.transient = True
    ctrl.dt = 0.0
    assert O.OracleCase(mesh, ctrl).pimple_run()[0] == 51
