"""Fixed small workloads for profiler captures, each exiting 0 on its own:

  python -m mixsolver_b200.prof_cases channel  # mixed form, 128x64x64 channel, 3 outer iterations
                                               # (L2-resident pressure system)
  python -m mixsolver_b200.prof_cases piso     # mixed form, 80^3 x 6 tets, 1 PISO step
                                               # (HBM-resident pressure system)
  python -m mixsolver_b200.prof_cases asm      # FP64 form of the channel, 2 outer iterations
                                               # (assembly kernels)

Each prints its solve counts and the run's device time. Library tuning keys
(mgpu_set_tuning) may follow as KEY=VALUE arguments, e.g.
  python -m mixsolver_b200.prof_cases asm gather_faces=1"""
from __future__ import annotations

import sys

from . import abi, cases, meshgen
from . import solver as S


def main(argv=None) -> int:
    argv = list(argv if argv is not None else sys.argv[1:])
    for kv in [a for a in argv if "=" in a]:
        k, v = kv.split("=", 1)
        S.set_tuning(k, int(v))
        argv.remove(kv)
    what = (argv or ["channel"])[0]
    if what in ("channel", "asm"):
        mesh, ctrl = cases.channel3d(128, 64, 64, seed=0, outer_max=10**6, order_fn=S.rcm_order,
                                     mom=abi.MOM_JACOBI, ppe=abi.PPE_ILU0)
        ctrl.lin_max = 1000
        ctrl.precision = abi.PREC_MIXED if what == "channel" else abi.PREC_FP64
        g = S.UnsCase(mesh, ctrl)
        ier, log = g.simple_run(3 if what == "channel" else 2)
        print(what, ier, [r["lin_it"][:4] for r in log], g.timing()["total_ms"])
        return 0 if ier == 0 else 1
    if what == "piso":
        n = int(argv[1]) if argv and len(argv) > 1 else 80
        mesh, ctrl = cases.tet_box(n, steps=10, ppe=abi.PPE_IC0, mom=abi.MOM_JACOBI)
        mesh = cases.rcm_renumber(mesh, S.rcm_order)
        ctrl.lin_tol = 1e-10
        ctrl.lin_max = 3000
        ctrl.precision = abi.PREC_MIXED
        u0 = meshgen.taylor_green(S.compute_geometry(mesh)["xc"], seed=0)
        g = S.UnsCase(mesh, ctrl)
        g.upload(u=u0)
        ier, log = g.piso_run(1)
        print(what, ier, [r["lin_it"][:5] for r in log], g.timing()["total_ms"], "bytes", g.device_bytes())
        return 0 if ier == 0 else 1
    print("usage: python -m mixsolver_b200.prof_cases channel|piso|asm", file=sys.stderr)
    return 2


if __name__ == "__main__":
    sys.exit(main())
