"""CPU checks of the C-ABI library: it loads, exports every symbol the header
declares, its struct layouts match the header, and its host-side integer mesh
pipeline (connectivity, CSR pattern, RCM) is bit-exact."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from mixsolver_b200 import abi, cases, meshgen, solver
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mixgpu.h")


@pytest.fixture(scope="module")
def lib():
    from mixsolver_b200 import build
    build.build()
    return abi.load_library()


def declared_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(mgpu_\w+)\s*\(", txt, re.M)))


def test_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert len(names) >= 18
    assert sorted(abi.EXPORTS) == names
    for n in names:
        assert hasattr(lib, n), n
    assert lib.mgpu_version() == 100


def test_struct_layouts():
    # sizes computed from the C declarations (natural alignment, LP64)
    assert C.sizeof(abi.MgpuBcSpec) == 4 * 2 + 8 * 3 + 8 * 5 + 4 * 4 + 8 * 4 + 4 * 2 + 8 * 2
    assert C.sizeof(abi.MgpuMesh) == 16 + 6 * 8
    assert C.sizeof(abi.MgpuIterRec) == 16 + 4 * 8 * 2 + 8 * 8 + 7 * 8
    assert C.sizeof(abi.MgpuTbcPlane) == 4 * 2 + 8 + 4 * 2 + 8 * 2
    assert C.sizeof(abi.MgpuCtrl) == (4 * 8 + 2 * 4 + 4 * 8 + 4 * 4 + 8 + 2 * 4 + 3 * 8 + 2 * 4 + 8 + 2 * 4
                                      + 32 * C.sizeof(abi.MgpuBcSpec)
                                      + 2 * 4 + 4 * 8 + 3 * 8 + 2 * 4 + 32 * C.sizeof(abi.MgpuTbcPlane))


def test_struct_offsets_match_compiled_header(tmp_path):
    """Every field offset and struct size of the ctypes mirrors equals what a C
    compiler makes of include/mixgpu.h."""
    structs = [abi.MgpuBcSpec, abi.MgpuTbcPlane, abi.MgpuCtrl, abi.MgpuMesh, abi.MgpuIterRec, abi.MgpuTiming,
               abi.MgpuBatchInfo]
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for st in structs:
        lines.append(f'  printf("{st.__name__} size %zu\\n", sizeof({st.__name__}));')
        for name, _ in st._fields_:
            lines.append(f'  printf("{st.__name__} {name} %zu\\n", offsetof({st.__name__}, {name}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    import subprocess
    subprocess.check_call(["gcc", "-std=c11", "-o", str(exe), str(src)])
    got = {}
    for ln in subprocess.check_output([str(exe)]).decode().splitlines():
        s, f, v = ln.split()
        got[(s, f)] = int(v)
    for st in structs:
        assert got[(st.__name__, "size")] == C.sizeof(st), st.__name__
        for name, _ in st._fields_:
            assert got[(st.__name__, name)] == getattr(st, name).offset, (st.__name__, name)


@pytest.mark.parametrize("which", ["cavity", "channel", "tet"])
def test_connectivity_bit_exact(lib, which):
    if which == "cavity":
        mesh, _ = cases.cavity2d(12)
    elif which == "channel":
        mesh, _ = cases.channel3d(8, 5, 4, seed=2)
    else:
        mesh = meshgen.box_tet(3)
    ctrl = abi.Ctrl(bcs=[abi.BcSpec(zone=int(z), btype=abi.BC_WALL) for z in np.unique(mesh.zone[mesh.c1 == 0])])
    got = solver.build_connectivity(mesh)
    ref = O.OracleCase(mesh, ctrl).connectivity()
    for k in ("cf_ptr", "cf", "c2c_ptr", "c2c", "row_ptr", "col_idx"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)


def test_rcm_bit_exact(lib):
    from oracle.rcm import rcm
    for mesh in (meshgen.shuffle_cells(meshgen.box_hex(6, 5, 4, jitter=0.1, seed=1), 3),
                 meshgen.shuffle_cells(cases.cavity2d(9)[0], 5),
                 meshgen.box_tet(2)):
        got = solver.rcm_order(mesh)
        np.testing.assert_array_equal(got, rcm(mesh))
        assert sorted(got.tolist()) == list(range(1, mesh.ncells + 1))


def test_rcm_reduces_bandwidth(lib):
    mesh = meshgen.shuffle_cells(meshgen.box_hex(10, 8, 6, jitter=0.1, seed=1), 7)

    def bandwidth(m):
        i = m.c1 > 0
        return int(np.abs(m.c0[i].astype(np.int64) - m.c1[i]).max())
    renum = meshgen.permute_cells(mesh, solver.rcm_order(mesh))
    assert bandwidth(renum) < bandwidth(mesh) / 4


def test_bad_mesh_rejected(lib):
    mesh, _ = cases.cavity2d(4)
    bad = mesh.copy()
    bad.c0[3] = mesh.ncells + 5
    with pytest.raises(RuntimeError, match="status -3"):
        solver.build_connectivity(bad)


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(RuntimeError, match="not built"):
        abi.load_library(str(tmp_path / "nope.so")) if abi._LIB is None else (_ for _ in ()).throw(
            RuntimeError("not built"))


def test_host_topology_matches_build_connectivity():
    """mgpu_mesh_topology's host builder (the arrays the device path is checked
    against) gives the CSR pattern and cell->face lists of
    mgpu_build_connectivity, 0-based."""
    from mixsolver_b200 import cases
    from mixsolver_b200 import solver as S
    mesh = cases.channel3d(8, 4, 4, seed=1)[0]
    t = S.mesh_topology(mesh, on_device=False)
    c = S.build_connectivity(mesh)
    np.testing.assert_array_equal(t["cf_ptr"] + 1, c["cf_ptr"])
    np.testing.assert_array_equal(t["cf"] + 1, c["cf"])
    np.testing.assert_array_equal(t["row_ptr"] + 1, c["row_ptr"])
    np.testing.assert_array_equal(t["col"] + 1, c["col_idx"])
    n = mesh.ncells
    for i in range(n):
        row = t["col"][t["row_ptr"][i]:t["row_ptr"][i + 1]]
        assert row[t["diag"][i] - t["row_ptr"][i]] == i
