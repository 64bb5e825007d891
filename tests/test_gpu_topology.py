"""The integer mesh pipeline and the RCM order built on the device, entry for
entry against the host builder (itself bit-exact with the reference's
build_connectivity / build_cell_csr, tests/test_abi_cpu.py) and against the
independent RCM restatement of the oracle (oracle/rcm.py). mgpu_case_create
builds its arrays this way."""
import numpy as np
import pytest

from mixsolver_b200 import cases, meshgen
from mixsolver_b200 import solver as S
from oracle.rcm import rcm as oracle_rcm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib(gpu_lib):
    return gpu_lib


def _meshes():
    yield "cavity16", cases.cavity2d(16)[0]
    yield "channel_shuffled", meshgen.sort_faces(meshgen.shuffle_cells(
        meshgen.box_hex(24, 12, 12, lx=4.0, jitter=0.1, seed=2, zones=(4, 5, 6, 6, 6, 6)), 3))
    yield "tets", meshgen.box_tet(6, wall_zone=4)
    yield "channel_rcm", cases.channel3d(32, 16, 16, seed=1, order_fn=S.rcm_order)[0]


@pytest.mark.parametrize("name,mesh", list(_meshes()), ids=[n for n, _ in _meshes()])
def test_device_topology_equals_host(name, mesh):
    dev = S.mesh_topology(mesh, on_device=True)
    host = S.mesh_topology(mesh, on_device=False)
    for k in host:
        np.testing.assert_array_equal(dev[k], host[k], err_msg=k)


@pytest.mark.parametrize("name,mesh", list(_meshes()), ids=[n for n, _ in _meshes()])
def test_device_rcm_equals_host_and_oracle(name, mesh):
    dev = S.rcm_order_device(mesh)
    np.testing.assert_array_equal(dev, S.rcm_order(mesh))
    np.testing.assert_array_equal(dev, oracle_rcm(mesh))


def test_device_pipeline_full_channel():
    """The measured workload's mesh: 128 x 64 x 64 hex, cells shuffled: the
    device RCM order and the device topology of the renumbered mesh equal the
    host's (524,288 cells, 1.59 M faces)."""
    mesh = meshgen.box_hex(128, 64, 64, lx=4.0, jitter=0.10, seed=0, zones=(4, 5, 6, 6, 6, 6))
    mesh = meshgen.shuffle_cells(mesh, 1)
    dev = S.rcm_order_device(mesh)
    np.testing.assert_array_equal(dev, S.rcm_order(mesh))
    m2 = meshgen.sort_faces(meshgen.permute_cells(mesh, dev))
    a, b = S.mesh_topology(m2, True), S.mesh_topology(m2, False)
    for k in b:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
