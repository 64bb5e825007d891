"""Batched runs: many resident cases advanced together (mgpu_batch_*).

* FP64 members: the batched assembly launches compute exactly what each
  case's own launches compute and the Krylov solves are the single-case
  kernels, so every member equals its own mgpu_simple_run / mgpu_piso_run bit
  for bit.
* Mixed-precision members: their Krylov phases run in the lane kernel. The
  mixed solves reduce over fixed row chunks, so their results do not depend
  on the number of blocks or on the other systems of a launch: every member
  equals its single-case mixed run bit for bit, alone or in any mix, under
  any lane policy.
"""
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
    n = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (n if n > 0 else 1.0)


def _cavities(prec, sizes=(6, 9, 12, 7), iters=12, re=(400.0, 1000.0, 150.0, 2000.0)):
    out = []
    for k, n in enumerate(sizes):
        mesh, ctrl = cases.cavity3d(n, re=re[k % len(re)], seed=k, outer_max=iters, mom=abi.MOM_JACOBI,
                                    ppe=abi.PPE_IC0)
        ctrl.precision = prec
        ctrl.lin_max = 2000
        out.append((mesh, ctrl))
    return out


def _single(mesh, ctrl, steps, piso=False, u0=None):
    g = S.UnsCase(mesh, ctrl)
    if u0 is not None:
        g.upload(u=u0)
    ier, log = g.piso_run(steps) if piso else g.simple_run(steps)
    return ier, log, g.fields()


def _batched(specs, modes, steps, policy=None, u0s=None):
    objs = []
    for k, (mesh, ctrl) in enumerate(specs):
        g = S.UnsCase(mesh, ctrl)
        if u0s is not None and u0s[k] is not None:
            g.upload(u=u0s[k])
        objs.append(g)
    B = S.CaseBatch(objs, policy=policy)
    nrec, ier = B.run(modes, steps)
    res = []
    for k, g in enumerate(objs):
        e, log = g.finish()
        assert e == ier[k]
        assert len(log) == nrec[k]
        res.append((int(ier[k]), log, g.fields()))
    info = B.info()
    B.close()
    return res, info


def test_fp64_batch_bit_identical_to_single_runs():
    specs = _cavities(abi.PREC_FP64, sizes=(5, 8, 6))
    got, info = _batched(specs, [0] * len(specs), 10)
    assert info["graph"] == 1, info
    for (mesh, ctrl), (ier, log, f) in zip(specs, got):
        ier1, log1, f1 = _single(mesh, copy.deepcopy(ctrl), 10)
        assert ier == ier1 == 0
        assert len(log) == len(log1) == 10
        for r, r1 in zip(log, log1):
            assert r["lin_it"] == r1["lin_it"]
            assert r["imbal"] == r1["imbal"] and r["du_max"] == r1["du_max"]
        for k in ("u", "p", "flux"):
            assert np.array_equal(f[k], f1[k]), k


def test_mixed_batch_bit_identical_to_single_mixed_runs():
    specs = _cavities(abi.PREC_MIXED)
    got, info = _batched(specs, [0] * len(specs), 12)
    assert info["autotuned"] == 1 and info["graph"] == 1, info
    assert info["launches_per_iter"] > 0
    for (mesh, ctrl), (ier, log, f) in zip(specs, got):
        ier1, log1, f1 = _single(mesh, copy.deepcopy(ctrl), 12)
        assert ier == ier1 == 0
        assert len(log) == len(log1)
        for r, r1 in zip(log, log1):
            assert all(e == 0 for e in r["lin_ierr"][:4]), r["lin_ierr"]
            assert all(x <= ctrl.lin_tol for x in r["lin_res"][:4]), r["lin_res"]
            assert r["lin_it"] == r1["lin_it"] and r["lin_res"] == r1["lin_res"]
        for k in ("u", "p", "flux"):
            assert np.array_equal(f[k], f1[k]), (k, rel(f[k], f1[k]))


@pytest.mark.parametrize("policy", [(64, 2), (32768, 1)])
def test_result_same_alone_and_in_the_mix(policy):
    """(64, 2): every member on one of two wide lanes; (32768, 1): every
    member on a single-block lane. Either way each member's result is the one
    it gets alone."""
    specs = _cavities(abi.PREC_MIXED, sizes=(9, 5, 11, 7), iters=8)
    mix, _ = _batched(specs, [0] * 4, 8, policy=policy)
    alone, _ = _batched([specs[2]], [0], 8, policy=(64, 4))
    for k in ("u", "p", "flux"):
        assert np.array_equal(mix[2][2][k], alone[0][2][k]), k
    assert [r["lin_it"] for r in mix[2][1]] == [r["lin_it"] for r in alone[0][1]]


def test_mixed_solve_independent_of_block_count():
    """The single-case mixed run on 1 block, on 2 blocks and on many blocks:
    the same fields bit for bit."""
    mesh, ctrl = cases.cavity3d(14, re=700.0, seed=2, outer_max=4, mom=abi.MOM_JACOBI)
    ctrl.precision = abi.PREC_MIXED
    ctrl.lin_max = 2000
    out = []
    try:
        for sbr, mb in ((1 << 20, 1), (0, 2), (0, 64)):
            S.set_tuning("single_block_rows", sbr)
            S.set_tuning("min_blocks", mb)
            out.append(_single(mesh, copy.deepcopy(ctrl), 4))
    finally:
        S.set_tuning("single_block_rows", 32768)
        S.set_tuning("min_blocks", 1)
    for ier, log, f in out[1:]:
        assert ier == out[0][0] == 0
        assert [r["lin_it"] for r in log] == [r["lin_it"] for r in out[0][1]]
        for k in ("u", "p", "flux"):
            assert np.array_equal(f[k], out[0][2][k]), k


def test_piso_and_simple_in_one_batch():
    mesh_t, ctrl_t = cases.tet_box(4, dt=1e-3, steps=4)
    ctrl_t.lin_max = 2000
    u0 = meshgen.taylor_green(O.OracleCase(mesh_t, ctrl_t).geometry()["xc"], seed=3)
    specs = _cavities(abi.PREC_FP64, sizes=(6,), iters=6) + [(mesh_t, ctrl_t)]
    got, _ = _batched(specs, [0, 1], 0, u0s=[None, u0])
    ier0, log0, f0 = _single(*specs[0], 6)
    ier1, log1, f1 = _single(mesh_t, copy.deepcopy(ctrl_t), 4, piso=True, u0=u0)
    assert got[0][0] == ier0 == 0 and got[1][0] == ier1 == 0
    assert len(got[0][1]) == 6 and len(got[1][1]) == 4
    for k in ("u", "p", "flux"):
        assert np.array_equal(got[0][2][k], f0[k]), k
        assert np.array_equal(got[1][2][k], f1[k]), k
    for r, r1 in zip(got[1][1], log1):
        assert r["t_now"] == r1["t_now"] and r["cfl_max"] == r1["cfl_max"]


def test_mixed_piso_batch_close_to_single():
    mesh, ctrl = cases.tet_box(4, dt=1e-3, steps=5)
    ctrl.lin_max = 2000
    ctrl.precision = abi.PREC_MIXED
    u0 = meshgen.taylor_green(O.OracleCase(mesh, ctrl).geometry()["xc"], seed=3)
    mesh2, ctrl2 = cases.tet_box(3, dt=1e-3, steps=5)
    ctrl2.lin_max = 2000
    ctrl2.precision = abi.PREC_MIXED
    u02 = meshgen.taylor_green(O.OracleCase(mesh2, ctrl2).geometry()["xc"], seed=5)
    got, _ = _batched([(mesh, ctrl), (mesh2, ctrl2)], [1, 1], 5, u0s=[u0, u02])
    _, _, f1 = _single(mesh, copy.deepcopy(ctrl), 5, piso=True, u0=u0)
    assert got[0][0] == 0
    for k in ("u", "p", "flux"):
        assert rel(got[0][2][k], f1[k]) < 1e-6, (k, rel(got[0][2][k], f1[k]))


def test_uneven_iteration_limits_and_rejected_run():
    """Members stop at their own limit; a PISO run the control rejects returns
    ier 30 and no records, as mgpu_piso_run does."""
    specs = _cavities(abi.PREC_MIXED, sizes=(5, 6, 7), iters=10)
    specs[1][1].outer_max = 4
    objs = [S.UnsCase(m, c) for m, c in specs]
    B = S.CaseBatch(objs)
    nrec, ier = B.run([0, 0, 1], 0)
    assert list(nrec) == [10, 4, 0]
    assert list(ier) == [0, 0, 30]
    assert list(B.poll()) == [1, 1, 1]
    B.close()


def test_step_and_poll_interface():
    specs = _cavities(abi.PREC_MIXED, sizes=(5, 7), iters=9)
    objs = [S.UnsCase(m, c) for m, c in specs]
    assert objs[0].begin(0, 3) == 0
    assert objs[1].begin(0) == 0
    B = S.CaseBatch(objs, policy=(16384, 8))
    assert B.step(2) == 2
    assert B.step(2) == 1          # the first member stopped at 3 iterations
    assert list(B.poll()) == [1, 0]
    assert B.step(10) == 0
    e0, l0 = objs[0].finish()
    e1, l1 = objs[1].finish()
    assert (e0, len(l0), e1, len(l1)) == (0, 3, 0, 9)
    B.close()


def test_launch_count_is_measured():
    """mgpu_batch_info's gpu_launches counts the kernels a batch runs: a CUDA
    graph replay adds the kernels it recorded, which equal the launches of one
    iteration launch by launch; each step adds its flag kernel."""
    specs = _cavities(abi.PREC_MIXED, sizes=(5, 7), iters=30)
    objs = [S.UnsCase(m, c) for m, c in specs]
    for g in objs:
        assert g.begin(0) == 0
    B = S.CaseBatch(objs, policy=(16384, 8))
    B.step(2)
    i0 = B.info()
    B.step(3)
    i1 = B.info()
    assert i1["graph"] == 1
    assert i1["gpu_launches"] - i0["gpu_launches"] == 3 * i1["launches_per_iter"] + 1
    B.close()
    for g in objs:
        g.finish()


def test_sized_lanes_keep_their_own_system():
    """Few big systems each get a lane sized by their work; with the capacity
    shrunk (block slots reserved) the narrow lanes are too small for the
    biggest system, which must still run on its own lane: every member equals
    its single-case run."""
    specs = []
    for k, n in enumerate((59, 39, 34)):
        mesh, ctrl = cases.cavity3d(n, re=600.0, seed=k, outer_max=3, mom=abi.MOM_JACOBI, ppe=abi.PPE_IC0)
        ctrl.precision = abi.PREC_MIXED
        ctrl.lin_max = 2000
        specs.append((mesh, ctrl))
    cap = S.batch_plan(np.array([59 ** 3, 39 ** 3, 34 ** 3], np.int32), 32768, 4, 16)[1]
    assert min(cap) < 7  # a lane narrower than the 59^3 system needs (7 blocks)
    S.set_tuning("batch_reserve_blocks", 256)
    try:
        got, _ = _batched(specs, [0, 0, 0], 3, policy=(32768, 4))
    finally:
        S.set_tuning("batch_reserve_blocks", 0)
    for (mesh, ctrl), (ier, log, f) in zip(specs, got):
        ier1, log1, f1 = _single(mesh, copy.deepcopy(ctrl), 3)
        assert ier == ier1 == 0
        for k in ("u", "p", "flux"):
            assert np.array_equal(f[k], f1[k]), k
