"""Shared by the fixture generator (make_golden.py) and the tests: the compact
mesh encoding of committed mesh fixtures, and the controls of the reference's
recorded cases that the fixtures reproduce."""
from __future__ import annotations

import os

import numpy as np

from mixsolver_b200.abi import (BC_MASSINLET, BC_OUTFLOW, BC_SYMMETRY, BC_WALL, MOM_ILU0, PPE_IC0, BcSpec,
                                Ctrl)
from mixsolver_b200.meshgen import FaceMesh

HERE = os.path.dirname(os.path.abspath(__file__))
LOWSPEED_MESH = os.path.join(HERE, "channel_lowspeed_mesh.npz")
LOWSPEED_PIN = os.path.join(HERE, "channel_lowspeed_pin.json")


def lowspeed_control(outer_max=8000):
    """cluster_cases/channel_lowspeed/unMesh.control: air at 300 K (rho 1.177,
    mu 1.846e-5), Re_H = 100; symmetry (zone 4), walls (zone 7), mass-flow
    inlet 1.8460e-4 (zone 5), outflow (zone 6); alpha_u 0.7, alpha_p 0.3,
    outer_tol 1e-10 (absolute), lin_tol 1e-8, lin_max 300, IC(0) pressure."""
    return Ctrl(rho=1.177, mu=1.846e-5, alpha_u=0.7, alpha_p=0.3, outer_max=outer_max, outer_tol=1.0e-10,
                lin_tol=1e-8, lin_max=300, conv_blend=0.0, nonorth_corr=1.0, ppe_precond=PPE_IC0,
                mom_solver=MOM_ILU0,
                bcs=[BcSpec(zone=4, btype=BC_SYMMETRY), BcSpec(zone=7, btype=BC_WALL),
                     BcSpec(zone=5, btype=BC_MASSINLET, mdot=1.8460e-4), BcSpec(zone=6, btype=BC_OUTFLOW)])


def encode_mesh(mesh) -> dict:
    """A face mesh as small integer streams, both steps exact: node coordinates
    as indexes into the sorted unique values of each axis, and every integer
    array as differences of consecutive entries."""
    out = {}
    for a, name in enumerate("xyz"):
        u = np.unique(mesh.x[:, a])
        idx = np.searchsorted(u, mesh.x[:, a])
        assert np.array_equal(u[idx], mesh.x[:, a])
        out["u" + name] = u
        out["i" + name] = np.diff(idx.astype(np.int64), prepend=0).astype(np.int32)
    for k in ("fnode_ptr", "fnodes", "c0", "c1", "zone"):
        out[k] = np.diff(getattr(mesh, k).astype(np.int64), prepend=0).astype(np.int32)
    out["ncells"] = np.array(mesh.ncells)
    return out


def decode_mesh(path: str) -> FaceMesh:
    g = np.load(path)
    cs = lambda a: np.cumsum(a.astype(np.int64)).astype(np.int32)
    x = np.stack([g["u" + n][cs(g["i" + n])] for n in "xyz"], axis=1)
    return FaceMesh(x=np.ascontiguousarray(x), fnode_ptr=cs(g["fnode_ptr"]), fnodes=cs(g["fnodes"]),
                    c0=cs(g["c0"]), c1=cs(g["c1"]), zone=cs(g["zone"]), ncells=int(g["ncells"]), zone_names={})
