"""The library's Fluent ASCII .cas reader (mgpu_cas_read) on the CPU: files
written here from generated meshes read back bit for bit, in every face-record
form the reader accepts (uniform face type, per-face type, polygon with a
count); the same arrays as the fixture reader; the reader's error codes. With
MIXSOLVER_REF naming a reference checkout, the reference's own 80x80 cavity
mesh reads the same through both readers."""
import os
import sys

import numpy as np
import pytest

from mixsolver_b200 import cases, meshgen
from mixsolver_b200 import solver as S

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
from casread import read_cas as fixture_read  # noqa: E402

# the reference checkout, when the environment names it (MIXSOLVER_REF)
_REF = os.environ.get("MIXSOLVER_REF", "")
REF_CAS = os.path.join(_REF, "cluster_cases/cavity_Re1000/unMesh.cas") if _REF else ""


def write_cas(mesh, path, form="uniform", polygon_every=0):
    """Fluent ASCII: (2 3), node, cell and face declarations and records (hex
    integers), one face record per run of faces of one zone, zone names."""
    nn, nf, nc = mesh.nnodes, mesh.nfaces, mesh.ncells
    out = ['(0 "written by the test")', "(2 3)", f"(10 (0 1 {nn:x} 0 3))", f"(10 (1 1 {nn:x} 1 3)("]
    out += [" ".join(repr(float(v)) for v in xyz) for xyz in mesh.x]
    out += ["))", f"(12 (0 1 {nc:x} 0))", f"(12 (7 1 {nc:x} 1 4))", f"(13 (0 1 {nf:x} 0))"]
    k = 0
    while k < nf:
        z = int(mesh.zone[k])
        e = k
        while e < nf and mesh.zone[e] == z:
            e += 1
        counts = mesh.fnode_ptr[k + 1:e + 1] - mesh.fnode_ptr[k:e]
        uniform = form == "uniform" and not polygon_every and len(set(counts.tolist())) == 1 and counts[0] <= 4
        ftype = int(counts[0]) if uniform else 0
        bc = 2 if mesh.c1[k] > 0 else 3
        out.append(f"(13 ({z:x} {k + 1:x} {e:x} {bc:x} {ftype:x})(")
        for f in range(k, e):
            nodes = mesh.fnodes[mesh.fnode_ptr[f]:mesh.fnode_ptr[f + 1]]
            words = []
            if not uniform:
                poly = polygon_every and f % polygon_every == 0
                words += ["5", f"{len(nodes):x}"] if poly or len(nodes) > 4 else [f"{len(nodes):x}"]
            words += [f"{int(v):x}" for v in nodes] + [f"{int(mesh.c0[f]):x}", f"{int(mesh.c1[f]):x}"]
            out.append(" ".join(words))
        out.append("))")
        k = e
    for z in sorted(set(mesh.zone.tolist())):
        out.append(f"(45 ({z} {mesh.zone_names.get(z, 'zone')} zone-{z})())")
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def same(a, b):
    assert a.ncells == b.ncells
    for k in ("x", "fnode_ptr", "fnodes", "c0", "c1", "zone"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)


def _named(mesh):
    mesh.zone_names = {int(z): ("interior" if z == 1 else f"wall{z}") for z in set(mesh.zone.tolist())}
    return mesh


@pytest.mark.parametrize("form,poly", [("uniform", 0), ("mixed", 0), ("mixed", 3)])
def test_round_trip_hex(tmp_path, form, poly):
    mesh = _named(cases.cavity2d(6)[0])
    p = tmp_path / "m.cas"
    write_cas(mesh, p, form, poly)
    got = S.read_cas(p)
    same(got, mesh)
    assert got.zone_names == mesh.zone_names
    same(fixture_read(str(p)), got)


def test_round_trip_tets(tmp_path):
    mesh = _named(meshgen.sort_faces(meshgen.box_tet(3, wall_zone=4)))
    p = tmp_path / "t.cas"
    write_cas(mesh, p, "mixed")
    same(S.read_cas(p), mesh)


def test_reader_errors(tmp_path):
    with pytest.raises(ValueError, match="ier 1"):
        S.read_cas(tmp_path / "missing.cas")
    mesh = _named(cases.cavity2d(4)[0])
    p = tmp_path / "bad.cas"
    write_cas(mesh, p, "mixed")
    text = p.read_text()
    # a node index past the node count
    p.write_text(text.replace(f"(10 (1 1 {mesh.nnodes:x} 1 3)(", f"(10 (1 1 {mesh.nnodes - 1:x} 1 3)(", 1)
                 .replace(f"(10 (0 1 {mesh.nnodes:x} 0 3))", f"(10 (0 1 {mesh.nnodes - 1:x} 0 3))", 1))
    with pytest.raises(ValueError, match="ier (7|21)"):
        S.read_cas(p)
    # an unknown face type
    lines = text.splitlines()
    i = next(k for k, ln in enumerate(lines) if ln.startswith("(13 (") and not ln.startswith("(13 (0 "))
    lines[i + 1] = "7 " + lines[i + 1].split(" ", 1)[1]
    p.write_text("\n".join(lines) + "\n")
    with pytest.raises(ValueError, match="ier 11"):
        S.read_cas(p)


@pytest.mark.skipif(not REF_CAS or not os.path.exists(REF_CAS), reason="MIXSOLVER_REF not set to a reference checkout")
def test_reference_mesh_reads_as_the_fixture_reader():
    got = S.read_cas(REF_CAS)
    assert (got.ncells, got.nfaces) == (6400, 25760)
    same(got, fixture_read(REF_CAS))
