"""The Fortran drop-in (mixsolver_b200/fortran/) against the C-ABI, on the CPU.

No Fortran compiler is available here, so the bind(C) module is checked
textually: each bind(C) derived type lists the fields of its C struct in the
same order (the ctypes mirror, itself checked against the compiled header by
test_abi_cpu.py), every bound name is an exported symbol of the library, and
the wrappers keep the argument lists of the reference's drivers."""
import os
import re

import pytest

from mixsolver_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
FDIR = os.path.join(os.path.dirname(HERE), "mixsolver_b200", "fortran")


def _src(name):
    return open(os.path.join(FDIR, name)).read()


def _type_fields(src, tname):
    m = re.search(r"type, bind\(C\), public :: %s\n(.*?)end type %s" % (tname, tname), src, re.S)
    assert m, tname
    names = []
    for line in m.group(1).splitlines():
        line = line.split("!")[0]
        if "::" not in line:
            continue
        decl = line.split("::", 1)[1]
        for item in re.split(r",(?![^(]*\))", decl):
            item = item.split("=")[0].strip()
            if item:
                names.append(re.sub(r"\(.*\)", "", item))
    return names


@pytest.mark.parametrize("tname,cstruct", [("mgpu_bc_spec", abi.MgpuBcSpec), ("mgpu_ctrl", abi.MgpuCtrl),
                                           ("mgpu_mesh", abi.MgpuMesh), ("mgpu_iter_rec", abi.MgpuIterRec)])
def test_bind_c_types_match_the_c_structs(tname, cstruct):
    assert _type_fields(_src("mod_gpu_iface.f90"), tname) == [f[0] for f in cstruct._fields_]


def test_bound_names_are_exported():
    lib = abi.load_library()
    names = re.findall(r"bind\(C, name='(\w+)'\)", _src("mod_gpu_iface.f90"))
    assert len(names) >= 13
    for n in names:
        assert hasattr(lib, n), n


def test_wrappers_keep_the_reference_argument_lists():
    src = _src("mod_uns_gpu.f90")
    assert re.search(r"subroutine simple_run_gpu\(m, conn, g, ctrl, bcs, fld, ier, nsteps\)", src)
    for name in ("piso_run_gpu", "pimple_run_gpu"):
        assert re.search(r"subroutine %s\(lm, hi, ctrl, bcs, fld, vtu_prefix, m_g, c_g, g_g, part, fld_g, ier\)"
                         % name, src)
