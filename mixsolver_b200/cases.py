"""The workloads this path is measured and checked on, as (mesh, ctrl) pairs.

Each builder returns a :class:`~mixsolver_b200.meshgen.FaceMesh` plus a
:class:`~mixsolver_b200.abi.Ctrl` equivalent to the ``.cas``/``.control`` pair the
reference would be given for the same run.
"""
from __future__ import annotations

import numpy as np

from . import meshgen
from .abi import (BC_POUTLET, BC_SYMMETRY, BC_VINLET_PARAB, BC_WALL, MOM_ILU0, MOM_JACOBI,
                  PPE_IC0, PPE_ILU0, BcSpec, Ctrl)


def cavity2d(n=64, mu=1.0e-3, outer_max=500, ppe=PPE_IC0, conv_blend=0.0, nonorth=1.0):
    """2-D lid-driven cavity (n x n x 1 hex, zones 4 symmetry / 5 wall, lid on
    the y = 1 plane of zone 5 at u = (1,0,0)); rho = 1, Re = 1/mu. The 64 x 64,
    mu = 1e-3, 500-iteration form is the CPU-runnable reference workload."""
    mesh = meshgen.cavity2d(n)
    ctrl = Ctrl(rho=1.0, mu=mu, alpha_u=0.7, alpha_p=0.3, outer_max=outer_max, outer_tol=0.0,
                lin_tol=1e-8, lin_max=200, conv_blend=conv_blend, nonorth_corr=nonorth,
                ppe_precond=ppe, mom_solver=MOM_ILU0,
                bcs=[BcSpec(zone=5, btype=BC_WALL, lid=(2, 1.0, (1.0, 0.0, 0.0))),
                     BcSpec(zone=4, btype=BC_SYMMETRY)])
    return mesh, ctrl


def rcm_renumber(mesh, order_fn):
    """Apply a cell ordering ``order_fn(mesh) -> new_of_old`` and re-sort faces."""
    new_of_old = order_fn(mesh)
    return meshgen.sort_faces(meshgen.permute_cells(mesh, new_of_old))


def channel3d(nx=128, ny=64, nz=64, seed=0, outer_max=200, order_fn=None, mu=5.0e-3,
              mom=MOM_JACOBI, ppe=PPE_ILU0):
    """3-D channel on [0,4]x[0,1]x[0,1]: interior nodes jittered +-10 % of the
    local spacing, cells shuffled (seeded) then renumbered by ``order_fn``
    (reverse Cuthill-McKee in the measured runs). Inlet x=0 parabolic in y
    (the reference's one-axis profile, Umean = 1), outlet x=4 pressure p = 0,
    no-slip walls; rho = 1, mu = 5e-3 (Re_h = 200)."""
    mesh = meshgen.box_hex(nx, ny, nz, lx=4.0, ly=1.0, lz=1.0, jitter=0.10, seed=seed,
                           zones=(4, 5, 6, 6, 6, 6))
    mesh = meshgen.shuffle_cells(mesh, seed + 1)
    if order_fn is not None:
        mesh = rcm_renumber(mesh, order_fn)
    else:
        mesh = meshgen.sort_faces(mesh)
    ctrl = Ctrl(rho=1.0, mu=mu, alpha_u=0.7, alpha_p=0.3, outer_max=outer_max, outer_tol=0.0,
                lin_tol=1e-8, lin_max=200, conv_blend=0.0, nonorth_corr=1.0,
                ppe_precond=ppe, mom_solver=mom,
                bcs=[BcSpec(zone=4, btype=BC_VINLET_PARAB, umean=1.0, uspan=1.0, uorigin=0.0, uaxis=2),
                     BcSpec(zone=5, btype=BC_POUTLET, pval=0.0),
                     BcSpec(zone=6, btype=BC_WALL)])
    return mesh, ctrl


def cavity3d(n=16, re=1000.0, seed=0, outer_max=100, jitter=0.10, ppe=PPE_IC0, mom=MOM_ILU0):
    """3-D lid-driven cube n^3 (jittered hex), lid y=1 moving at u=(1,0,0),
    rho = 1, mu = 1/Re."""
    mesh = meshgen.box_hex(n, n, n, jitter=jitter, seed=seed, zones=(5, 5, 5, 5, 5, 5))
    mesh = meshgen.sort_faces(mesh)
    ctrl = Ctrl(rho=1.0, mu=1.0 / re, alpha_u=0.7, alpha_p=0.3, outer_max=outer_max, outer_tol=0.0,
                lin_tol=1e-8, lin_max=200, ppe_precond=ppe, mom_solver=mom,
                bcs=[BcSpec(zone=5, btype=BC_WALL, lid=(2, 1.0, (1.0, 0.0, 0.0)))])
    return mesh, ctrl


def tet_box(n=80, dt=1.0e-3, steps=100, mu=1.0e-3, ppe=PPE_IC0, mom=MOM_ILU0):
    """n^3 hexes on the unit cube, each split into 6 tets; no-slip walls;
    transient PISO (dt, 2 correctors, implicit Euler). The Taylor-Green initial
    field comes from :func:`meshgen.taylor_green` at the cell centres."""
    mesh = meshgen.box_tet(n, wall_zone=4)
    ctrl = Ctrl(rho=1.0, mu=mu, outer_max=1, lin_tol=1e-8, lin_max=200, ppe_precond=ppe,
                mom_solver=mom, transient=True, time_scheme=1, dt=dt, n_time_max=steps,
                n_correct=2, bcs=[BcSpec(zone=4, btype=BC_WALL)])
    return mesh, ctrl
