"""Serving on the GPU: a stream of SIMPLE and PISO requests served with
continuous batching; every result equals the one the same request gets when
served alone (mixed precision: the lane solves do not depend on the lane;
FP64: single-case solvers), bit for bit."""
import dataclasses
import math

import numpy as np
import pytest

from mixsolver_b200 import abi, cases, meshgen, serve
from mixsolver_b200 import solver as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib(gpu_lib):
    return gpu_lib


def _stream(prec):
    reqs = []
    specs = [(0, 7, 400.0), (1, 3, 500.0), (0, 5, 1500.0), (0, 9, 100.0), (1, 4, 2000.0), (0, 6, 800.0)]
    for k, (mode, n, re) in enumerate(specs):
        if mode == 0:
            mesh, ctrl = cases.cavity3d(n, re=re, seed=k, outer_max=30, mom=abi.MOM_JACOBI, ppe=abi.PPE_IC0)
            u0 = None
            steps = 12
        else:
            mesh, ctrl = cases.tet_box(n, dt=1e-3, steps=6, mu=1.0 / re)
            u0 = meshgen.taylor_green(S.compute_geometry(mesh)["xc"], seed=k)
            steps = 5
        ctrl.precision = prec
        ctrl.lin_max = 2000
        reqs.append(serve.Request(rid=k, arrival=0.002 * k, mode=mode, mesh=mesh, ctrl=ctrl, nsteps=steps, u0=u0))
    return reqs


def _fresh(r):
    return dataclasses.replace(r, admitted=math.nan, finished=math.nan, ier=-1, nrec=0, fields=None, error=None)


@pytest.mark.parametrize("prec", [abi.PREC_MIXED, abi.PREC_FP64])
def test_served_results_equal_results_served_alone(prec):
    reqs = _stream(prec)
    srv = serve.Server(serve.GpuBackend(policy=(4096, 2)), budget_bytes=2e9, active_cells=2000, tick_iters=3,
                       keep_fields=True)
    out = srv.run([_fresh(r) for r in reqs])
    assert srv.batches_built > 1  # the active set changed while requests came and went
    for r in out:
        assert r.error is None and r.ier == 0, (r.rid, r.error, r.ier)
        assert r.nrec == r.nsteps
        alone = serve.Server(serve.GpuBackend(policy=(4096, 2)), budget_bytes=2e9, tick_iters=3,
                             keep_fields=True).run([_fresh(reqs[r.rid])])[0]
        assert alone.nrec == r.nrec and alone.ier == r.ier
        for k in ("u", "p", "flux"):
            assert np.array_equal(alone.fields[k], r.fields[k]), (r.rid, k)
    s = serve.summary(out, wall=max(r.finished for r in out))
    assert s["completed"] == len(reqs) and s["p99_s"] >= s["p50_s"] > 0
