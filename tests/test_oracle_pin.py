"""The CPU oracle against the reference's own published outputs and against
the committed golden fixtures (tests/golden/make_golden.py)."""
import hashlib
import json
import os

import numpy as np
import pytest

from mixsolver_b200 import cases
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def oracle_sha():
    return hashlib.sha256(open(os.path.join(ROOT, "oracle", "oracle.cpp"), "rb").read()).hexdigest()[:16]


def test_ghia_pin_matches_published():
    """Steady SIMPLE of the oracle on the reference's own 80x80 / 40x40 cavity
    meshes and control reproduces the published centre-line L2 errors
    (2.897e-2 stated to 4 digits in cluster_cases/cavity_Re1000/unMesh.control,
    9.12e-2 to 3 digits in cluster_cases/README.md:190)."""
    pin = json.load(open(os.path.join(GOLD, "ghia_pin.json")))
    assert pin["oracle_sha"] == oracle_sha(), "oracle changed: rerun tests/golden/make_golden.py"
    runs = {r["mesh"]: r for r in pin["runs"]}
    r80 = runs["cluster_cases/cavity_Re1000/unMesh.cas"]
    assert r80["ier"] == 0 and r80["outer_iterations"] == 1000
    assert abs(r80["ghia_l2"] - 2.897e-2) < 0.5e-5          # 4 significant digits
    assert r80["final_imbal"] < 1e-15                        # mass conserved to round-off
    r40 = runs["cases/natconv/cavity.cas"]
    assert abs(r40["ghia_l2"] - 9.12e-2) / 9.12e-2 < 5e-3    # 3 significant digits


def test_pimple_pin_matches_published_history():
    """PIMPLE of the oracle on the reference's 80x80 cavity mesh, dt 0.01, 2
    outer iterations x 2 corrections per step, to t = 10, against the history
    that cluster_cases/cavity_Re1000/README.md section 4 records for the
    reference's own run (MPI np = 4; its transient control was not kept in the
    case, alpha_u 0.7 is taken from the case's control): max|u| at t = 10 to 4
    digits, the 5 s means of max|u| to 0.5 %, those of du/dt and the
    centre-line L2 at t = 10 to 3 %."""
    pin = json.load(open(os.path.join(GOLD, "ghia_pin.json")))
    assert pin["oracle_sha"] == oracle_sha(), "oracle changed: rerun tests/golden/make_golden.py"
    r = pin["pimple"]
    pub = r["published"]
    assert r["ier"] == 0 and r["steps"] == 1000
    assert abs(r["umax_t10"] - pub["umax_t10"]) < 0.5e-4
    for got, want in zip(r["umax_mean"], pub["umax_mean"]):
        assert abs(got - want) / want < 5e-3
    for got, want in zip(r["dudt_mean"], pub["dudt_mean"]):
        assert abs(got - want) / want < 3e-2
    assert abs(r["ghia_l2_t10"] - pub["ghia_l2_t10"]) / pub["ghia_l2_t10"] < 3e-2


def _hist(log):
    return (np.array([r["lin_it"] for r in log]), np.array([r["lin_res"] for r in log]),
            np.array([r["imbal"] for r in log]), np.array([r["du_max"] for r in log]))


def test_oracle_matches_golden_cases():
    g = np.load(os.path.join(GOLD, "oracle_cases.npz"))
    assert str(g["oracle_sha"]) == oracle_sha(), "oracle changed: rerun tests/golden/make_golden.py"
    m, c = cases.cavity2d(16, outer_max=30)
    oc = O.OracleCase(m, c)
    ier, log = oc.simple_run()
    assert ier == 0 and len(log) == 30
    it, res, imb, du = _hist(log)
    np.testing.assert_array_equal(it, g["cav16_lin_it"])
    np.testing.assert_array_equal(res, g["cav16_lin_res"])
    f = oc.fields()
    np.testing.assert_array_equal(f["u"], g["cav16_u"])
    np.testing.assert_array_equal(f["flux"], g["cav16_flux"])
    m, c = cases.channel3d(12, 6, 6, seed=3, outer_max=10)
    oc = O.OracleCase(m, c)
    ier, log = oc.simple_run()
    it, res, imb, du = _hist(log)
    np.testing.assert_array_equal(it, g["chan_lin_it"])
    np.testing.assert_array_equal(oc.fields()["u"], g["chan_u"])


def test_nan_scan_semantics():
    """nan_scan ordering of test_nan_guard.f90:72-121: lowest cell wins, then
    field order u_x, u_y, u_z, p; NaN vs Inf labelled; clean field set finite."""
    m, c = cases.cavity2d(8, outer_max=1)
    oc = O.OracleCase(m, c)
    n = m.ncells
    kc1, kc2 = n // 2 + 1, max(1, n // 4)
    u = np.zeros((n, 3)); p = np.zeros(n)
    oc.upload(u=u, p=p)
    assert oc.nan_scan()[0] == 0
    u[kc1 - 1, 1] = np.nan
    oc.upload(u=u)
    ifin, field, cell, val, kind = oc.nan_scan()
    assert (ifin, field, cell, kind) == (1, 2, kc1, 1)
    u[kc1 - 1, 1] = 0.0
    p[kc2 - 1] = np.inf
    oc.upload(u=u, p=p)
    ifin, field, cell, val, kind = oc.nan_scan()
    assert (ifin, field, cell, kind) == (1, 4, kc2, 2)
    # lower cell index dominates the field order
    u[kc1 - 1, 0] = np.inf
    p[kc2 - 1] = np.nan
    oc.upload(u=u, p=p)
    ifin, field, cell, val, kind = oc.nan_scan()
    assert (ifin, field, cell) == (1, 4, kc2)
    u[:] = 0.0; p[:] = 0.0
    oc.upload(u=u, p=p)
    assert oc.nan_scan()[0] == 0


def test_krylov_contracts():
    """ierr/it contracts of mod_uns_linsolver.f90: homogeneous rhs returns x=0,
    it=0; maxit leaves it = maxit (BiCGStab) or maxit+1 (CG); a zero pivot is a
    factorisation failure (+10); a matrix without diagonal breaks cg_jacobi."""
    rp = np.array([1, 3, 5], np.int32); ci = np.array([1, 2, 1, 2], np.int32)
    v = np.array([4.0, -1.0, -1.0, 3.0])
    x, it, res, ierr = O.krylov_solve(rp, ci, v, np.zeros(2), np.ones(2), 1e-8, 10, 2)
    assert (it, ierr) == (0, 0) and np.all(x == 0)
    b = np.array([1.0, 2.0])
    x, it, res, ierr = O.krylov_solve(rp, ci, v, b, np.zeros(2), 1e-12, 10, 1)
    assert ierr == 0 and res <= 1e-12
    np.testing.assert_allclose(v.reshape(2, 2) @ x, b, rtol=1e-12)
    # maxit semantics on a larger SPD system
    m, c = cases.cavity2d(16, outer_max=1)
    n = 60
    A = np.diag(np.full(n, 2.0)) - np.diag(np.ones(n - 1), 1) - np.diag(np.ones(n - 1), -1)
    rows, cols = np.nonzero(A)
    rp = np.concatenate([[0], np.cumsum(np.bincount(rows, minlength=n))]).astype(np.int32) + 1
    ci = (cols + 1).astype(np.int32)
    vals = A[rows, cols]
    bb = np.linspace(1, 2, n)
    _, it, _, ierr = O.krylov_solve(rp, ci, vals, bb, np.zeros(n), 1e-14, 3, 1)
    assert (it, ierr) == (4, 1)
    _, it, _, ierr = O.krylov_solve(rp, ci, vals, bb, np.zeros(n), 1e-14, 3, 3)
    assert (it, ierr) == (3, 1)
    # zero pivot in ILU(0) -> ierr = 12
    v0 = v.copy(); v0[0] = 0.0
    _, it, _, ierr = O.krylov_solve(np.array([1, 3, 5], np.int32), np.array([1, 2, 1, 2], np.int32), v0,
                                    np.array([1.0, 1.0]), np.zeros(2), 1e-8, 10, 0)
    assert ierr == 12
    # missing diagonal -> cg_jacobi breakdown (ierr = 2)
    _, it, _, ierr = O.krylov_solve(np.array([1, 2, 3], np.int32), np.array([2, 1], np.int32),
                                    np.array([1.0, 1.0]), np.array([1.0, 1.0]), np.zeros(2), 1e-8, 10, 1)
    assert ierr == 2


def test_norm2_scaled():
    a = np.array([3.0, 4.0])
    assert O.norm2(a) == 5.0
    big = np.array([1e200, 1e200])
    assert np.isfinite(O.norm2(big)) and abs(O.norm2(big) / (np.sqrt(2) * 1e200) - 1) < 1e-15


# --- the reference's recorded channel run (cluster_cases/channel_lowspeed) ---
import sys  # noqa: E402

sys.path.insert(0, GOLD)
from fixtures import LOWSPEED_MESH, LOWSPEED_PIN, decode_mesh, lowspeed_control  # noqa: E402


def test_channel_lowspeed_first_iteration_is_the_reference_log():
    """cluster_cases/channel_lowspeed/README.md section 4 records the reference
    binary's first outer iteration on this mesh and control as
    `it=1: mass-imbal = 5.113E-13, du_max = 2.840E-04, lin-it = 278` (bit for
    bit the same as an archived log). The oracle prints the same line: the
    same numbers in the same es10.3 format and the same iteration count. The
    case uses the mass-flow inlet, the outflow rescale, walls and symmetry."""
    mesh = decode_mesh(LOWSPEED_MESH)
    assert (mesh.ncells, mesh.nfaces, mesh.nnodes) == (30000, 120400, 60802)
    oc = O.OracleCase(mesh, lowspeed_control())
    ier, log = oc.simple_run(1)
    assert ier == 0
    r = log[0]
    assert f"{r['imbal']:.3E}" == "5.113E-13"
    assert f"{r['du_max']:.3E}" == "2.840E-04"
    assert r["itl_max"] == 278


def test_channel_lowspeed_convergence_is_the_reference_log():
    """The oracle's full run on the same case (tests/golden/make_golden.py):
    `CONVERGED after 773` with du_max 9.950E-11, as the README records for the
    reference binary."""
    pin = json.load(open(LOWSPEED_PIN))
    assert pin["oracle_sha"] == oracle_sha(), "oracle changed: rerun tests/golden/make_golden.py"
    pub = pin["published"]
    assert pin["ier"] == 0
    assert pin["converged_after"] == pub["converged_after"] == 773
    assert f"{pin['final_du_max']:.3E}" == pub["final_du_max"]
    assert f"{pin['it1']['imbal']:.3E}" == pub["it1_imbal"]
    assert pin["it1"]["itl_max"] == pub["it1_lin_it"]


@pytest.mark.slow
@pytest.mark.skipif(not os.environ.get("MIXSOLVER_SLOW"), reason="set MIXSOLVER_SLOW=1 (about 4 min of CPU)")
def test_channel_lowspeed_full_run_reproduces_pin():
    mesh = decode_mesh(LOWSPEED_MESH)
    oc = O.OracleCase(mesh, lowspeed_control())
    ier, log = oc.simple_run(logcap=8000)
    pin = json.load(open(LOWSPEED_PIN))
    assert ier == 0 and len(log) == pin["converged_after"] == 773
    assert log[-1]["du_max"] == pin["final_du_max"]


from fixtures import (NATCONV_MESH, NATCONV_PIN, natconv_control, natconv_initial_T,  # noqa: E402
                      nusselt)


def test_natconv_ra1e4_is_the_reference_result():
    """The energy equation with Boussinesq buoyancy: the oracle on the
    reference's own Rayleigh-Benard case (cases/natconv/cavity.cas with
    fluid/rb_Ra1e4.control: 40 x 40 cavity, hot bottom / cold top through
    tbc_plane lines, conv_blend 1, the driver's perturbed initial T) converges
    after 2245 outer iterations with Nu = 2.1601, as cases/natconv/README.md
    section 3 records for the reference binary (run here in full, about 16 s)."""
    mesh = decode_mesh(NATCONV_MESH)
    assert mesh.ncells == 1600
    ctrl = natconv_control()
    oc = O.OracleCase(mesh, ctrl)
    geo = oc.geometry()
    oc.upload_T(natconv_initial_T(mesh, geo["xc"]))
    ier, log = oc.simple_run(logcap=20000)
    T, _ = oc.temperature()
    nu = nusselt(mesh, geo, T, ctrl)
    pin = json.load(open(NATCONV_PIN))
    assert pin["oracle_sha"] == oracle_sha(), "oracle changed: rerun tests/golden/make_golden.py"
    assert ier == 0 and len(log) == pin["converged_after"] == pin["published"]["converged_after"] == 2245
    assert f"{nu:.4f}" == pin["published"]["nusselt"] == "2.1601"
    assert nu == pin["nusselt"]
    assert log[-1]["dT_max"] < ctrl.outer_tol and log[-1]["du_max"] < ctrl.outer_tol
