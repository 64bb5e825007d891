"""The synthetic meshes every workload is built from, checked on the CPU with
the oracle's geometry (compute_geometry restated): every cell closed (its
outward face-area vectors sum to zero), positive volumes filling the box, face
orientation from c0 to c1, and the shapes the workloads name (config 3:
n^3 x 6 tets)."""
import numpy as np
import pytest

from mixsolver_b200 import cases, meshgen
from oracle import oracle as O


def _check(mesh, ctrl, box_volume):
    o = O.OracleCase(mesh, ctrl)
    g = o.geometry()
    N = mesh.ncells
    c0 = mesh.c0 - 1
    c1 = mesh.c1 - 1
    closure = np.zeros((N, 3))
    np.add.at(closure, c0, g["sf"])
    inner = c1 >= 0
    np.add.at(closure, c1[inner], -g["sf"][inner])
    scale = np.abs(g["sf"]).max()
    assert np.abs(closure).max() < 1e-12 * max(scale, 1.0) * 10, np.abs(closure).max()
    assert (g["vol"] > 0).all()
    assert abs(g["vol"].sum() - box_volume) < 1e-9 * box_volume
    # the area vector of an interior face points from its owner to its neighbour
    d = g["xc"][c1[inner]] - g["xc"][c0[inner]]
    assert ((d * g["sf"][inner]).sum(1) > 0).all()
    return g


@pytest.mark.parametrize("n", [3, 5])
def test_tet_box(n):
    mesh, ctrl = cases.tet_box(n)
    assert mesh.ncells == 6 * n ** 3
    # 2 F_i + F_b = 4 N (each tet has 4 faces); F_b = 2 triangles per boundary square
    nint = mesh.n_interior()
    assert 2 * nint + (mesh.nfaces - nint) == 4 * mesh.ncells
    assert mesh.nfaces - nint == 12 * n * n
    _check(mesh, ctrl, 1.0)


def test_jittered_hex_cavity():
    mesh, ctrl = cases.cavity3d(6, seed=3)
    _check(mesh, ctrl, 1.0)


def test_channel_after_shuffle_and_rcm():
    from oracle.rcm import rcm
    mesh, ctrl = cases.channel3d(8, 4, 4, seed=1, order_fn=rcm)
    assert mesh.ncells == 128
    _check(mesh, ctrl, 4.0)


def test_cavity2d_layout():
    mesh, ctrl = cases.cavity2d(8)
    assert mesh.ncells == 64
    zones = set(mesh.zone[mesh.c1 == 0].tolist())
    assert zones == {4, 5}   # symmetry planes and the walls, as the reference's gen_cas layout
    vol = O.OracleCase(mesh, ctrl).geometry()["vol"]
    g = _check(mesh, ctrl, float(vol.sum()))
    np.testing.assert_allclose(g["vol"], vol[0], rtol=1e-12)   # a uniform grid
