"""Regenerate the committed golden fixtures under tests/golden/.

Run from the repository root with MIXSOLVER_REF naming a checkout of the
reference project:

    MIXSOLVER_REF=<reference checkout> python tests/golden/make_golden.py

Produces
  * ghia_pin.json -- the oracle's steady SIMPLE on the reference's own cavity
    meshes (cluster_cases/cavity_Re1000/unMesh.cas, 80x80; cases/natconv/cavity.cas,
    40x40) with the control of cluster_cases/cavity_Re1000/unMesh.control, scored
    with the centre-line probe of mod_uns_output.f90:246-350. The Ghia table is
    read from the reference source at generation time; only the resulting L2
    is stored. The reference publishes 2.897e-2 (80x80, unMesh.control:63,
    cluster_cases/README.md:189) and 9.12e-2 (40x40, cluster_cases/README.md:190).
    It also holds the oracle's PIMPLE run on the 80x80 mesh to t = 10, against
    the transient history that cluster_cases/cavity_Re1000/README.md section 4
    records (np = 4, dt = 0.01, 2 x 2 corrections per step).
  * channel_lowspeed_mesh.npz, channel_lowspeed_pin.json -- the reference's
    recorded channel case (cluster_cases/channel_lowspeed: mass-flow inlet,
    outflow, walls, symmetry) as a compact mesh fixture, and the oracle's run
    to convergence on it beside the iteration line and convergence count its
    README records for the reference binary.
  * natconv_cavity_mesh.npz, natconv_ra1e4_pin.json -- the reference's
    Rayleigh-Benard case at Ra = 1e4 (cases/natconv, 40 x 40 cavity with the
    energy equation and Boussinesq buoyancy) as a compact mesh fixture, and
    the oracle's run to convergence beside the iteration count and Nusselt
    number its README records.
  * oracle_cases.npz -- oracle histories and final fields on small synthetic
    workloads (the same generators the CUDA tests use), used by the CPU suite
    to detect any change in the oracle's results.
The oracle source hash is stored in each fixture so a stale fixture is caught.
"""
from __future__ import annotations

import hashlib
import json
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from casread import read_cas  # noqa: E402
from fixtures import (LOWSPEED_MESH, LOWSPEED_PIN, NATCONV_MESH, NATCONV_PIN, decode_mesh,  # noqa: E402
                      encode_mesh, lowspeed_control, mirror_asymmetry, natconv_control, natconv_initial_T,
                      nusselt)
from mixsolver_b200 import cases  # noqa: E402
from mixsolver_b200.abi import (BC_SYMMETRY, BC_WALL, MOM_ILU0, MOM_JACOBI, PPE_IC0, PPE_JACOBI,  # noqa: E402
                                BcSpec, Ctrl)
from oracle import oracle as O  # noqa: E402

REF = os.environ.get("MIXSOLVER_REF", "")


def oracle_hash() -> str:
    return hashlib.sha256(open(os.path.join(ROOT, "oracle", "oracle.cpp"), "rb").read()).hexdigest()[:16]


def ghia_table():
    src = open(os.path.join(REF, "src/unstructured/mod_uns_output.f90")).read()

    def arr(name):
        mm = re.search(name + r"\s*=\s*\[(.*?)\]", src, re.S)
        return np.array([float(v.replace("_dp", "")) for v in mm.group(1).replace("&", " ").split(",")])
    return arr("yg"), arr("u1000")


def probe_l2(xc, u, yg, uref):
    """probe_velocity (8 nearest centroids, w = 1/(d^2+1e-12)) at (0.5, y, 0.5)
    and the relative L2 over the 15 interior stations, as ghia_compare does."""
    num = den = 0.0
    for i, (y, ur) in enumerate(zip(yg, uref)):
        d2 = ((xc - np.array([0.5, y, 0.5])) ** 2).sum(1)
        idx = np.argsort(d2, kind="stable")[:8]
        w = 1.0 / (d2[idx] + 1e-12)
        uq = (w[:, None] * u[idx]).sum(0) / w.sum()
        if 0 < i < len(yg) - 1:
            num += (uq[0] - ur) ** 2
            den += ur * ur
    return float(np.sqrt(num / den))


def cavity_control(outer_max):
    # cluster_cases/cavity_Re1000/unMesh.control
    return Ctrl(rho=1.0, mu=0.001, alpha_u=0.7, alpha_p=0.3, outer_max=outer_max, outer_tol=0.0,
                lin_tol=1e-8, lin_max=300, conv_blend=1.0, nonorth_corr=0.0, ppe_precond=PPE_IC0,
                mom_solver=MOM_ILU0,
                bcs=[BcSpec(zone=5, btype=BC_WALL, lid=(2, 1.0, (1.0, 0.0, 0.0))),
                     BcSpec(zone=4, btype=BC_SYMMETRY)])


def make_ghia():
    yg, u1000 = ghia_table()
    out = {"oracle_sha": oracle_hash(), "runs": []}
    for rel, iters, published in (("cluster_cases/cavity_Re1000/unMesh.cas", 1000, 2.897e-2),
                                  ("cases/natconv/cavity.cas", 3000, 9.12e-2)):
        mesh = read_cas(os.path.join(REF, rel))
        oc = O.OracleCase(mesh, cavity_control(iters))
        ier, log = oc.simple_run(logcap=iters)
        xc = oc.geometry()["xc"]
        u = oc.fields()["u"]
        out["runs"].append(dict(mesh=rel, ncells=mesh.ncells, outer_iterations=len(log), ier=ier,
                                ghia_l2=probe_l2(xc, u, yg, u1000), published_l2=published,
                                final_imbal=log[-1]["imbal"], final_du_max=log[-1]["du_max"],
                                it1=log[0]))
        print(rel, out["runs"][-1]["ghia_l2"])
    make_pimple_pin(out)
    with open(os.path.join(ROOT, "tests/golden/ghia_pin.json"), "w") as f:
        json.dump(out, f, indent=1)


def make_pimple_pin(out):
    """PIMPLE (pimple_run_mpi at one rank) on the reference's 80x80 cavity mesh
    with its control and the recorded transient settings (dt 0.01, 2 outer
    iterations x 2 corrections per step; cluster_cases/cavity_Re1000/README.md
    section 4), 1000 steps to t = 10 in one run: the centre-line L2, max|u| at
    t = 10, and the 500-step means of max|u| and du/dt that the README tabulates
    for t = 0-5 and 5-10."""
    yg, u1000 = ghia_table()
    mesh = read_cas(os.path.join(REF, "cluster_cases/cavity_Re1000/unMesh.cas"))
    c = cavity_control(1)
    c.transient = True
    c.dt = 0.01
    c.n_time_max = 1000
    c.n_outer_iter = 2
    c.n_correct = 2
    oc = O.OracleCase(mesh, c)
    xc = oc.geometry()["xc"]
    ier, log = oc.pimple_run(1000, logcap=1000)
    u = oc.fields()["u"]
    du = np.array([r["du_max"] for r in log])
    um = np.array([r["umax"] for r in log])
    out["pimple"] = dict(mesh="cluster_cases/cavity_Re1000/unMesh.cas", steps=len(log), ier=ier,
                         ghia_l2_t10=probe_l2(xc, u, yg, u1000),
                         umax_t10=float(np.sqrt((u ** 2).sum(1)).max()),
                         umax_mean=[float(um[:500].mean()), float(um[500:].mean())],
                         dudt_mean=[float(du[:500].mean()), float(du[500:].mean())],
                         itl_max=[int(min(r["itl_max"] for r in log)), int(max(r["itl_max"] for r in log))],
                         published=dict(ghia_l2_t10=4.51e-1, umax_t10=0.8996, umax_mean=[0.8718, 0.9003],
                                        dudt_mean=[5.174e-1, 1.054e-1]))
    print("pimple", out["pimple"]["ghia_l2_t10"], out["pimple"]["umax_t10"])


def make_lowspeed():
    """The reference's recorded channel run (cluster_cases/channel_lowspeed:
    README.md section 4 logs it=1 mass-imbal 5.113E-13, du_max 2.840E-04,
    lin-it 278, and CONVERGED after 773): its mesh as a compact fixture, plus
    the oracle's full run to convergence on it."""
    mesh = read_cas(os.path.join(REF, "cluster_cases/channel_lowspeed/unMesh.cas"))
    np.savez_compressed(LOWSPEED_MESH, **encode_mesh(mesh))
    assert np.array_equal(decode_mesh(LOWSPEED_MESH).x, mesh.x)
    oc = O.OracleCase(mesh, lowspeed_control())
    ier, log = oc.simple_run(logcap=8000)
    last = log[-1]
    out = dict(oracle_sha=oracle_hash(), mesh="cluster_cases/channel_lowspeed/unMesh.cas", ier=ier,
               converged_after=len(log), final_du_max=last["du_max"], final_imbal=last["imbal"],
               it1=dict(imbal=log[0]["imbal"], du_max=log[0]["du_max"], itl_max=log[0]["itl_max"]),
               published=dict(it1_imbal="5.113E-13", it1_du_max="2.840E-04", it1_lin_it=278,
                              converged_after=773, archived_converged_after=790, final_du_max="9.950E-11"))
    with open(LOWSPEED_PIN, "w") as f:
        json.dump(out, f, indent=1)
    print("lowspeed: converged after", len(log), "du_max", last["du_max"])


def make_natconv():
    """The reference's Rayleigh-Benard case at Ra = 1e4 (cases/natconv:
    cavity.cas, fluid/rb_Ra1e4.control; README.md section 3 records 2245
    iterations and Nu = 2.1601 on this 40 x 40 mesh): its mesh as a compact
    fixture, plus the oracle's run to convergence on it (the driver's initial
    temperature, thermal_wall_report's Nusselt number)."""
    mesh = read_cas(os.path.join(REF, "cases/natconv/cavity.cas"))
    np.savez_compressed(NATCONV_MESH, **encode_mesh(mesh))
    assert np.array_equal(decode_mesh(NATCONV_MESH).x, mesh.x)
    ctrl = natconv_control()
    oc = O.OracleCase(mesh, ctrl)
    geo = oc.geometry()
    oc.upload_T(natconv_initial_T(mesh, geo["xc"]))
    ier, log = oc.simple_run(logcap=20000)
    T, _ = oc.temperature()
    nu = nusselt(mesh, geo, T, ctrl)
    # The initial temperature is symmetric about the mid-plane x = L/2; the
    # reference's single roll grows from the asymmetric errors of its
    # direction-dependent ILU(0) momentum and temperature solves. With Jacobi
    # (mirror-invariant) solves the same case settles on the symmetric
    # two-roll branch instead.
    jc = natconv_control()
    jc.mom_solver, jc.ppe_precond = MOM_JACOBI, PPE_JACOBI
    oj = O.OracleCase(mesh, jc)
    oj.upload_T(natconv_initial_T(mesh, geo["xc"]))
    ier_j, log_j = oj.simple_run(logcap=20000)
    Tj, _ = oj.temperature()
    out = dict(oracle_sha=oracle_hash(), mesh="cases/natconv/cavity.cas", ier=ier, converged_after=len(log),
               nusselt=nu, T_min=float(T.min()), T_max=float(T.max()),
               asymmetry=mirror_asymmetry(mesh, geo["xc"], T),
               head=[dict(it=r["it"], lin_it=list(r["lin_it"][:5]), dT_max=r["dT_max"], du_max=r["du_max"])
                     for r in log[:5]],
               published=dict(converged_after=2245, nusselt="2.1601"),
               jacobi_branch=dict(solvers="BiCGStab+Jacobi momentum and temperature, PCG+Jacobi pressure",
                                  ier=ier_j, converged_after=len(log_j), nusselt=nusselt(mesh, geo, Tj, jc),
                                  asymmetry=mirror_asymmetry(mesh, geo["xc"], Tj)))
    with open(NATCONV_PIN, "w") as f:
        json.dump(out, f, indent=1)
    print("natconv: converged after", len(log), "Nu", nu, "; Jacobi solves:", len(log_j), "Nu",
          out["jacobi_branch"]["nusselt"])


def hist_arrays(log):
    return dict(lin_it=np.array([r["lin_it"] for r in log], np.int32),
                lin_res=np.array([r["lin_res"] for r in log]),
                imbal=np.array([r["imbal"] for r in log]),
                du_max=np.array([r["du_max"] for r in log]))


def make_cases():
    data = {"oracle_sha": np.array(oracle_hash())}
    # 2-D cavity, 16x16, 30 SIMPLE iterations (reference solvers)
    m, c = cases.cavity2d(16, outer_max=30)
    oc = O.OracleCase(m, c)
    ier, log = oc.simple_run()
    f = oc.fields()
    for k, v in hist_arrays(log).items():
        data[f"cav16_{k}"] = v
    data["cav16_u"], data["cav16_p"], data["cav16_flux"] = f["u"], f["p"], f["flux"]
    # small jittered channel, 10 iterations, BiCGStab+Jacobi / PCG+ILU(0)
    m, c = cases.channel3d(12, 6, 6, seed=3, outer_max=10)
    oc = O.OracleCase(m, c)
    ier, log = oc.simple_run()
    f = oc.fields()
    for k, v in hist_arrays(log).items():
        data[f"chan_{k}"] = v
    data["chan_u"], data["chan_p"] = f["u"], f["p"]
    np.savez_compressed(os.path.join(ROOT, "tests/golden/oracle_cases.npz"), **data)
    print("oracle_cases.npz written")


if __name__ == "__main__":
    only = "--lowspeed-only" in sys.argv or "--natconv-only" in sys.argv
    if not only:
        make_cases()
    if os.path.isdir(REF):
        if not only:
            make_ghia()
        if "--natconv-only" not in sys.argv:
            make_lowspeed()
        make_natconv()
    else:
        print("MIXSOLVER_REF not set to a reference checkout; ghia_pin.json, the channel_lowspeed and the "
              "natconv fixtures left unchanged")
