"""ctypes mirror of include/mixgpu.h and loader of the in-tree CUDA library.

The structures here are byte-for-byte the C structs of ``include/mixgpu.h``;
``Ctrl``/``BcSpec`` are the Python-side spelling of the reference's ``ctrl_t`` and
``bc_spec_t`` (``src/unstructured/mod_uns_control.f90:114-280``) with the same
defaults.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmixgpu.so")

# boundary types, mod_uns_control.f90:32-56
BC_WALL, BC_SYMMETRY, BC_VINLET, BC_POUTLET, BC_FARFIELD = 1, 2, 3, 4, 5
BC_SLIPWALL, BC_MASSINLET, BC_OUTFLOW, BC_INTERFACE, BC_VINLET_PARAB = 6, 7, 8, 9, 10
BC_NAMES = {"wall": BC_WALL, "symmetry": BC_SYMMETRY, "velocity-inlet": BC_VINLET,
            "pressure-outlet": BC_POUTLET, "pressure-far-field": BC_FARFIELD,
            "slip-wall": BC_SLIPWALL, "mass-flow-inlet": BC_MASSINLET,
            "outflow": BC_OUTFLOW, "velocity-inlet-parabolic": BC_VINLET_PARAB}

PPE_JACOBI, PPE_IC0, PPE_ILU0 = 0, 1, 2
MOM_ILU0, MOM_JACOBI = 0, 1
PREC_FP64, PREC_MIXED, PREC_FP64_POLY = 0, 1, 2
MAXBC = 32
MAXSOLVE = 8

# Krylov method ids of mgpu_krylov_solve
KRY_BICGSTAB_ILU0, KRY_CG_JACOBI, KRY_CG_IC0, KRY_BICGSTAB_JACOBI, KRY_CG_ILU0 = 0, 1, 2, 3, 4


class MgpuBcSpec(C.Structure):
    _fields_ = [("zone", C.c_int32), ("btype", C.c_int32), ("uvel", C.c_double * 3),
                ("pval", C.c_double), ("mdot", C.c_double), ("umean", C.c_double),
                ("uspan", C.c_double), ("uorigin", C.c_double), ("uaxis", C.c_int32),
                ("has_lid", C.c_int32), ("lid_dir", C.c_int32), ("pad0", C.c_int32),
                ("lid_coord", C.c_double), ("lid_vel", C.c_double * 3), ("ttype", C.c_int32),
                ("pad1", C.c_int32), ("tval", C.c_double), ("qval", C.c_double)]


MAXTBC = 32


class MgpuTbcPlane(C.Structure):
    _fields_ = [("bc", C.c_int32), ("pdir", C.c_int32), ("pcoord", C.c_double), ("ttype", C.c_int32),
                ("pad0", C.c_int32), ("tval", C.c_double), ("qval", C.c_double)]


class MgpuCtrl(C.Structure):
    _fields_ = [("rho", C.c_double), ("mu", C.c_double), ("alpha_u", C.c_double),
                ("alpha_p", C.c_double), ("outer_max", C.c_int32), ("lin_max", C.c_int32),
                ("outer_tol", C.c_double), ("lin_tol", C.c_double), ("conv_blend", C.c_double),
                ("nonorth_corr", C.c_double), ("ppe_precond", C.c_int32), ("mom_solver", C.c_int32),
                ("transient", C.c_int32), ("time_scheme", C.c_int32), ("dt", C.c_double),
                ("n_time_max", C.c_int32), ("n_correct", C.c_int32), ("body_force", C.c_double * 3),
                ("inlet_ramp", C.c_int32), ("precision", C.c_int32), ("mixed_tol", C.c_double),
                ("nbc", C.c_int32), ("n_outer_iter", C.c_int32), ("bc", MgpuBcSpec * MAXBC),
                ("energy", C.c_int32), ("boussinesq", C.c_int32), ("cp", C.c_double), ("k_cond", C.c_double),
                ("tref", C.c_double), ("beta", C.c_double), ("gravity", C.c_double * 3), ("ntbc", C.c_int32),
                ("pad_e", C.c_int32), ("tbc", MgpuTbcPlane * MAXTBC)]


class MgpuMesh(C.Structure):
    _fields_ = [("nnodes", C.c_int32), ("nfaces", C.c_int32), ("ncells", C.c_int32),
                ("pad0", C.c_int32), ("x", C.POINTER(C.c_double)),
                ("fnode_ptr", C.POINTER(C.c_int32)), ("fnodes", C.POINTER(C.c_int32)),
                ("c0", C.POINTER(C.c_int32)), ("c1", C.POINTER(C.c_int32)),
                ("zone", C.POINTER(C.c_int32))]


class MgpuIterRec(C.Structure):
    _fields_ = [("it", C.c_int32), ("itl_max", C.c_int32), ("nsolve", C.c_int32),
                ("pad0", C.c_int32), ("lin_it", C.c_int32 * MAXSOLVE),
                ("lin_ierr", C.c_int32 * MAXSOLVE), ("lin_res", C.c_double * MAXSOLVE),
                ("imbal", C.c_double), ("du_max", C.c_double), ("dT_max", C.c_double),
                ("ressum", C.c_double), ("umax", C.c_double), ("cfl_max", C.c_double),
                ("t_now", C.c_double)]


class MgpuTiming(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("spmv_launches", C.c_int64), ("spmv_ms", C.c_double),
                ("krylov_launches", C.c_int64), ("krylov_ms", C.c_double),
                ("gpu_launches", C.c_int64)]


class MgpuBatchInfo(C.Structure):
    _fields_ = [("ncases", C.c_int32), ("split_rows", C.c_int32), ("wide_lanes", C.c_int32),
                ("autotuned", C.c_int32), ("graph", C.c_int32), ("lanes", C.c_int32), ("blocks", C.c_int32),
                ("launches_per_iter", C.c_int32), ("tune_ms", C.c_double), ("step_ms", C.c_double),
                ("iters", C.c_int64), ("phase_ms", C.c_double * 8), ("asm_ms", C.c_double),
                ("lane_max_ms", C.c_double), ("lane_mean_ms", C.c_double), ("profiled_iters", C.c_int64),
                ("gpu_launches", C.c_int64)]


@dataclasses.dataclass
class BcSpec:
    """One ``bc`` control line (bc_spec_t)."""
    zone: int
    btype: int
    uvel: Sequence[float] = (0.0, 0.0, 0.0)
    pval: float = 0.0
    mdot: float = 0.0
    umean: float = 0.0
    uspan: float = 0.0
    uorigin: float = 0.0
    uaxis: int = 2
    lid: Optional[tuple] = None      # (dir, coord, (u, v, w)), the `lid` control line
    ttype: int = 0                   # thermal type (walls, outlets): 0 adiabatic, 1 fixed T, 2 fixed flux
    tval: float = 0.0
    qval: float = 0.0


@dataclasses.dataclass
class Ctrl:
    """ctrl_t defaults (mod_uns_control.f90:148-280) plus this library's options."""
    rho: float = 1.0
    mu: float = 0.01
    alpha_u: float = 0.7
    alpha_p: float = 0.3
    outer_max: int = 2000
    outer_tol: float = 1.0e-6
    lin_tol: float = 1.0e-8
    lin_max: int = 200
    conv_blend: float = 0.0
    nonorth_corr: float = 1.0
    ppe_precond: int = PPE_IC0
    mom_solver: int = MOM_ILU0
    transient: bool = False
    time_scheme: int = 1
    dt: float = 0.0
    n_time_max: int = 0
    n_correct: int = 2
    n_outer_iter: int = 1
    body_force: Sequence[float] = (0.0, 0.0, 0.0)
    inlet_ramp: int = 1
    precision: int = PREC_FP64
    mixed_tol: float = 1.0e-4
    bcs: list = dataclasses.field(default_factory=list)
    # energy equation (ctrl_t phase-10 fields): solved when energy is set
    energy: bool = False
    boussinesq: bool = False
    cp: float = 1005.0
    k_cond: float = 0.026
    tref: float = 0.0
    beta: float = 0.0
    gravity: Sequence[float] = (0.0, 0.0, 0.0)
    # tbc_plane lines: (bc index, dir 1-3, coord, ttype, tval, qval)
    tbc: list = dataclasses.field(default_factory=list)

    def to_c(self) -> MgpuCtrl:
        c = MgpuCtrl()
        for name in ("rho", "mu", "alpha_u", "alpha_p", "outer_tol", "lin_tol", "conv_blend",
                     "nonorth_corr", "dt", "mixed_tol"):
            setattr(c, name, float(getattr(self, name)))
        for name in ("outer_max", "lin_max", "ppe_precond", "mom_solver", "time_scheme",
                     "n_time_max", "n_correct", "n_outer_iter", "inlet_ramp", "precision"):
            setattr(c, name, int(getattr(self, name)))
        c.transient = 1 if self.transient else 0
        for k in range(3):
            c.body_force[k] = float(self.body_force[k])
        if len(self.bcs) > MAXBC:
            raise ValueError("too many bc lines")
        c.nbc = len(self.bcs)
        for i, b in enumerate(self.bcs):
            s = c.bc[i]
            s.zone, s.btype = int(b.zone), int(b.btype)
            for k in range(3):
                s.uvel[k] = float(b.uvel[k])
            s.pval, s.mdot = float(b.pval), float(b.mdot)
            s.umean, s.uspan, s.uorigin, s.uaxis = float(b.umean), float(b.uspan), float(b.uorigin), int(b.uaxis)
            if b.lid is not None:
                s.has_lid, s.lid_dir, s.lid_coord = 1, int(b.lid[0]), float(b.lid[1])
                for k in range(3):
                    s.lid_vel[k] = float(b.lid[2][k])
            s.ttype, s.tval, s.qval = int(b.ttype), float(b.tval), float(b.qval)
        c.energy = 1 if self.energy else 0
        c.boussinesq = 1 if self.boussinesq else 0
        c.cp, c.k_cond, c.tref, c.beta = float(self.cp), float(self.k_cond), float(self.tref), float(self.beta)
        for k in range(3):
            c.gravity[k] = float(self.gravity[k])
        if len(self.tbc) > MAXTBC:
            raise ValueError("too many tbc_plane lines")
        c.ntbc = len(self.tbc)
        for i, (bi, pdir, pc, tt, tv, qv) in enumerate(self.tbc):
            t = c.tbc[i]
            t.bc, t.pdir, t.pcoord, t.ttype, t.tval, t.qval = int(bi), int(pdir), float(pc), int(tt), float(tv), float(qv)
        return c


class MeshArrays:
    """Keeps the numpy arrays alive behind an MgpuMesh struct."""

    def __init__(self, m):
        self.x = np.ascontiguousarray(m.x, np.float64)
        self.fnode_ptr = np.ascontiguousarray(m.fnode_ptr, np.int32)
        self.fnodes = np.ascontiguousarray(m.fnodes, np.int32)
        self.c0 = np.ascontiguousarray(m.c0, np.int32)
        self.c1 = np.ascontiguousarray(m.c1, np.int32)
        self.zone = np.ascontiguousarray(m.zone, np.int32)
        s = MgpuMesh()
        s.nnodes, s.nfaces, s.ncells = self.x.shape[0], self.c0.shape[0], int(m.ncells)
        s.x = self.x.ctypes.data_as(C.POINTER(C.c_double))
        s.fnode_ptr = self.fnode_ptr.ctypes.data_as(C.POINTER(C.c_int32))
        s.fnodes = self.fnodes.ctypes.data_as(C.POINTER(C.c_int32))
        s.c0 = self.c0.ctypes.data_as(C.POINTER(C.c_int32))
        s.c1 = self.c1.ctypes.data_as(C.POINTER(C.c_int32))
        s.zone = self.zone.ctypes.data_as(C.POINTER(C.c_int32))
        self.struct = s


def dptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def records_to_list(recs, n: int) -> list:
    out = []
    for r in recs[:n]:
        ns = r.nsolve
        out.append(dict(it=r.it, itl_max=r.itl_max, nsolve=ns, lin_it=list(r.lin_it[:ns]),
                        lin_ierr=list(r.lin_ierr[:ns]), lin_res=list(r.lin_res[:ns]),
                        imbal=r.imbal, du_max=r.du_max, dT_max=r.dT_max, ressum=r.ressum,
                        umax=r.umax, cfl_max=r.cfl_max, t_now=r.t_now))
    return out


# Every symbol include/mixgpu.h declares (checked by the CPU test suite).
EXPORTS = ["mgpu_version", "mgpu_last_error", "mgpu_set_device", "mgpu_case_create",
           "mgpu_case_destroy", "mgpu_case_device_bytes", "mgpu_fields_upload",
           "mgpu_fields_download", "mgpu_simple_run_fields", "mgpu_simple_run", "mgpu_piso_run", "mgpu_pimple_run", "mgpu_nan_scan",
           "mgpu_krylov_solve", "mgpu_csr_matvec", "mgpu_build_connectivity", "mgpu_geometry",
           "mgpu_rcm_order", "mgpu_case_stage", "mgpu_cg_jacobi_noalloc", "mgpu_set_tuning", "mgpu_get_tuning",
           "mgpu_case_solve_times", "mgpu_case_timing", "mgpu_case_set_profiling", "mgpu_case_begin",
           "mgpu_case_finish", "mgpu_batch_create", "mgpu_batch_destroy", "mgpu_batch_set_policy",
           "mgpu_batch_step", "mgpu_batch_poll", "mgpu_batch_run", "mgpu_batch_info", "mgpu_batch_plan",
           "mgpu_batch_set_profiling", "mgpu_cas_read", "mgpu_cas_zone_names", "mgpu_cas_free",
           "mgpu_rcm_order_device", "mgpu_mesh_topology", "mgpu_interface_set", "mgpu_interface_set_T", "mgpu_interface_mode",
           "mgpu_interface_extract", "mgpu_pcg_poly_solve", "mgpu_temperature_upload",
           "mgpu_temperature_download"]
NOALLOC_MAX_ROWS = 131072

_LIB = None


def load_library(path: str = LIB_PATH):
    """Load the in-tree libmixgpu.so. Raises if it is missing: there is no
    fallback implementation."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise RuntimeError(f"libmixgpu.so not built at {path}; run __graft_entry__.build() "
                           "or python -m mixsolver_b200.build")
    lib = C.CDLL(path)
    P = C.POINTER
    i32p, dblp = P(C.c_int32), P(C.c_double)
    lib.mgpu_version.restype = C.c_int
    lib.mgpu_last_error.restype = C.c_char_p
    lib.mgpu_set_device.argtypes = [C.c_int]
    lib.mgpu_case_create.argtypes = [P(MgpuMesh), P(MgpuCtrl), P(C.c_void_p), P(C.c_int)]
    lib.mgpu_case_destroy.argtypes = [C.c_void_p]
    lib.mgpu_case_device_bytes.argtypes = [C.c_void_p, P(C.c_int64)]
    lib.mgpu_fields_upload.argtypes = [C.c_void_p, dblp, dblp, dblp, dblp, dblp]
    lib.mgpu_fields_download.argtypes = [C.c_void_p, dblp, dblp, dblp, dblp, dblp, dblp]
    lib.mgpu_simple_run.argtypes = [C.c_void_p, C.c_int, P(MgpuIterRec), C.c_int, P(C.c_int), P(C.c_int)]
    lib.mgpu_simple_run_fields.argtypes = [C.c_void_p, C.c_int, P(MgpuIterRec), C.c_int, P(C.c_int), P(C.c_int),
                                           dblp, dblp, dblp, dblp, dblp, dblp]
    lib.mgpu_piso_run.argtypes = [C.c_void_p, C.c_int, P(MgpuIterRec), C.c_int, P(C.c_int), P(C.c_int)]
    lib.mgpu_pimple_run.argtypes = [C.c_void_p, C.c_int, P(MgpuIterRec), C.c_int, P(C.c_int), P(C.c_int)]
    lib.mgpu_cas_read.argtypes = [C.c_char_p, P(MgpuMesh), P(C.c_void_p), P(C.c_int)]
    lib.mgpu_cas_zone_names.argtypes = [C.c_void_p, C.c_char_p, C.c_int, P(C.c_int)]
    lib.mgpu_cas_free.argtypes = [C.c_void_p]
    lib.mgpu_nan_scan.argtypes = [C.c_void_p, P(C.c_int), P(C.c_int), P(C.c_int), dblp, P(C.c_int)]
    lib.mgpu_krylov_solve.argtypes = [C.c_int, i32p, i32p, dblp, dblp, dblp, C.c_double, C.c_int,
                                      C.c_int, C.c_int, P(C.c_int), dblp, P(C.c_int)]
    lib.mgpu_temperature_upload.argtypes = [C.c_void_p, dblp, dblp, dblp]
    lib.mgpu_temperature_download.argtypes = [C.c_void_p, dblp, dblp]
    lib.mgpu_pcg_poly_solve.argtypes = [C.c_int, i32p, i32p, dblp, dblp, dblp, C.c_double, C.c_int,
                                        C.c_int, C.c_int, P(C.c_int), dblp, P(C.c_int)]
    lib.mgpu_csr_matvec.argtypes = [C.c_int, i32p, i32p, dblp, dblp, dblp]
    lib.mgpu_build_connectivity.argtypes = [P(MgpuMesh), i32p, i32p, i32p, i32p, i32p, i32p, i32p]
    lib.mgpu_geometry.argtypes = [P(MgpuMesh), dblp, dblp, dblp, dblp, dblp, dblp]
    lib.mgpu_rcm_order.argtypes = [P(MgpuMesh), i32p]
    lib.mgpu_rcm_order_device.argtypes = [P(MgpuMesh), i32p]
    lib.mgpu_interface_set.argtypes = [C.c_void_p, C.c_int, i32p, dblp, dblp]
    lib.mgpu_interface_mode.argtypes = [C.c_void_p, C.c_int]
    lib.mgpu_interface_set_T.argtypes = [C.c_void_p, C.c_int, i32p, dblp, dblp, i32p]
    lib.mgpu_interface_extract.argtypes = [C.c_void_p, C.c_int, i32p, dblp, dblp, dblp, P(C.c_int)]
    lib.mgpu_mesh_topology.argtypes = [P(MgpuMesh), C.c_int] + [i32p] * 12
    lib.mgpu_case_stage.argtypes = [C.c_void_p, C.c_int, C.c_int, dblp, dblp, dblp, dblp, dblp]
    lib.mgpu_cg_jacobi_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_double, C.c_int, C.c_int, C.c_void_p, P(C.c_int), dblp,
                                           P(C.c_int)]
    lib.mgpu_set_tuning.argtypes = [C.c_char_p, C.c_int]
    lib.mgpu_get_tuning.argtypes = [C.c_char_p, P(C.c_int)]
    lib.mgpu_case_solve_times.argtypes = [C.c_void_p, dblp, C.c_int, P(C.c_int)]
    lib.mgpu_case_timing.argtypes = [C.c_void_p, P(MgpuTiming)]
    lib.mgpu_case_set_profiling.argtypes = [C.c_void_p, C.c_int]
    lib.mgpu_case_begin.argtypes = [C.c_void_p, C.c_int, C.c_int, P(C.c_int)]
    lib.mgpu_case_finish.argtypes = [C.c_void_p, P(MgpuIterRec), C.c_int, P(C.c_int), P(C.c_int)]
    lib.mgpu_batch_create.argtypes = [P(C.c_void_p), C.c_int, P(C.c_void_p)]
    lib.mgpu_batch_destroy.argtypes = [C.c_void_p]
    lib.mgpu_batch_set_policy.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.mgpu_batch_step.argtypes = [C.c_void_p, C.c_int, P(C.c_int)]
    lib.mgpu_batch_poll.argtypes = [C.c_void_p, P(C.c_int)]
    lib.mgpu_batch_run.argtypes = [C.c_void_p, P(C.c_int), C.c_int, P(C.c_int), P(C.c_int)]
    lib.mgpu_batch_info.argtypes = [C.c_void_p, P(MgpuBatchInfo)]
    lib.mgpu_batch_set_profiling.argtypes = [C.c_void_p, C.c_int]
    lib.mgpu_batch_plan.argtypes = [C.c_int, i32p, dblp, C.c_int, C.c_int, C.c_int, i32p, i32p, P(C.c_int)]
    _LIB = lib
    return lib


def check(lib, rc: int, what: str):
    if rc != 0:
        msg = lib.mgpu_last_error()
        raise RuntimeError(f"{what} failed with status {rc}: {msg.decode() if msg else ''}")
