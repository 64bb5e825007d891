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
NATCONV_MESH = os.path.join(HERE, "natconv_cavity_mesh.npz")
NATCONV_PIN = os.path.join(HERE, "natconv_ra1e4_pin.json")


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


def natconv_control(outer_max=10000):
    """cases/natconv/fluid/rb_Ra1e4.control: Rayleigh-Benard at Ra = 1e4 on
    the 40 x 40 x 1 cavity, Pr 0.71 (rho = cp = 1, mu 1.523e-3, k 2.146e-3),
    Boussinesq with beta 3.33e-3, T_ref 300.5, g = (0, -9.81, 0); the wall
    zone 5 hot (301 K) at y = 0 and cold (300 K) at y = 1 through two
    tbc_plane lines, adiabatic elsewhere; symmetry zone 4; alpha_u 0.7,
    alpha_p 0.3, outer_tol 1e-6, lin_tol 1e-8, lin_max 400, conv_blend 1,
    no non-orthogonal correction, IC(0) pressure."""
    return Ctrl(rho=1.0, mu=1.523e-3, alpha_u=0.7, alpha_p=0.3, outer_max=outer_max, outer_tol=1.0e-6,
                lin_tol=1e-8, lin_max=400, conv_blend=1.0, nonorth_corr=0.0, ppe_precond=PPE_IC0,
                mom_solver=MOM_ILU0, energy=True, boussinesq=True, cp=1.0, k_cond=2.146e-3, beta=3.33e-3,
                tref=300.5, gravity=(0.0, -9.81, 0.0),
                bcs=[BcSpec(zone=5, btype=BC_WALL), BcSpec(zone=4, btype=BC_SYMMETRY)],
                tbc=[(0, 2, 0.0, 1, 301.0, 0.0), (0, 2, 1.0, 1, 300.0, 0.0)])


def natconv_initial_T(mesh, xc, init_T=300.5, t_pert=0.02):
    """The reference driver's initial temperature (mod_uns_driver.f90:182-196):
    init_T + t_pert sin(pi (x_c - x_min) / L_x), x over the mesh nodes."""
    xmin, xmax = float(mesh.x[:, 0].min()), float(mesh.x[:, 0].max())
    lx = max(xmax - xmin, np.finfo(float).eps)
    return init_T + t_pert * np.sin(np.arccos(-1.0) * (xc[:, 0] - xmin) / lx)


def nusselt(mesh, geo, T, ctrl):
    """thermal_wall_report (mod_uns_output.f90:365-475) for two fixed-T planes
    on one axis: Q = sum k area / dw (T_face - T_P) over each plane's faces,
    Nu = |Q_hot| / A_hot * L / (k dT)."""
    planes = [t for t in ctrl.tbc if t[3] == 1]
    tol = 1.0e-4 * float(np.max(mesh.x.max(0) - mesh.x.min(0)))
    res = []
    for (_, pdir, pc, _, tv, _) in planes:
        Q = A = 0.0
        for f in range(mesh.nfaces):
            if mesh.c1[f] != 0 or abs(geo["xf"][f, pdir - 1] - pc) > tol:
                continue
            c = mesh.c0[f] - 1
            dw = np.linalg.norm(geo["xf"][f] - geo["xc"][c])
            Q += ctrl.k_cond * geo["area"][f] / dw * (tv - T[c])
            A += geo["area"][f]
        res.append((tv, pc, Q, A))
    (th, ph, qh, ah), (tc, pcd, _, _) = sorted(res, key=lambda r: -r[0])
    return abs(qh) / ah * abs(ph - pcd) / (ctrl.k_cond * (th - tc))


def mirror_asymmetry(mesh, xc, T):
    """max |T(x, y) - T(x_min + x_max - x, y)| over the cell pairs that mirror
    each other across the cavity's vertical mid-plane: 0 for the symmetric
    two-roll state the driver's symmetric initial temperature leads to in exact
    arithmetic, O(dT) for a single roll."""
    xs = float(mesh.x[:, 0].min() + mesh.x[:, 0].max())
    key = {(round(x * 1e6), round(y * 1e6)): i for i, (x, y) in enumerate(xc[:, :2])}
    worst = 0.0
    for i, (x, y) in enumerate(xc[:, :2]):
        j = key.get((round((xs - x) * 1e6), round(y * 1e6)))
        if j is not None:
            worst = max(worst, abs(float(T[i]) - float(T[j])))
    return worst
