"""Host-side mirror of the reference's unstructured-solver module interface.

The names and argument meanings follow the Fortran modules this library
replaces, so a caller of the reference finds the same operations:

* :class:`UnsCase` -- ``uns_solver_init`` / ``uns_solver_step``
  (``src/unstructured/mod_uns_driver.f90:60-255``): a case built from a mesh and a
  control, kept resident on the GPU; :meth:`UnsCase.simple_run` is ``simple_run``
  (``mod_uns_simple.f90:88-288``) and :meth:`UnsCase.piso_run` is ``piso_run_mpi`` at
  one rank (``mod_uns_simple_mpi.f90:298-571``). Both return the reference's ``ier``.
* :func:`bicgstab_ilu0`, :func:`cg_jacobi`, :func:`cg_ic0` and :func:`csr_matvec`
  -- ``mod_uns_linsolver.f90``: ``(A, b, x, tol, maxit) -> (x, it, res, ierr)``.
* :func:`build_connectivity`, :func:`compute_geometry` -- the mesh pipeline.
* :class:`CaseBatch` -- no counterpart in the reference (one case per process
  there): many resident cases advanced together, each assembly kernel one
  launch over all of them and each Krylov phase one persistent launch.

Every call runs on the GPU through ``libmixgpu.so``; there is no CPU path and a
missing library raises.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi
from .abi import MeshArrays, MgpuBatchInfo, MgpuIterRec, MgpuTiming, dptr, iptr, records_to_list


def _lib():
    return abi.load_library()


class UnsCase:
    """One unstructured case resident in HBM (mesh, matrices, fields)."""

    def __init__(self, mesh, ctrl, device: int = 0):
        lib = _lib()
        abi.check(lib, lib.mgpu_set_device(int(device)), "mgpu_set_device")
        self.mesh = mesh
        self.ctrl = ctrl
        self._arrays = MeshArrays(mesh)
        self._cctrl = ctrl.to_c()
        self.h = C.c_void_p()
        ier = C.c_int(0)
        rc = lib.mgpu_case_create(C.byref(self._arrays.struct), C.byref(self._cctrl), C.byref(self.h),
                                  C.byref(ier))
        if rc != 0:
            msg = lib.mgpu_last_error().decode()
            raise RuntimeError(f"mgpu_case_create failed (status {rc}, ier {ier.value}): {msg}")
        self.N, self.F = mesh.ncells, mesh.nfaces

    def close(self):
        if self.h:
            _lib().mgpu_case_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, u=None, p=None, flux=None, u_old=None, u_old_old=None):
        conv = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        u, p, flux, u_old, u_old_old = map(conv, (u, p, flux, u_old, u_old_old))
        lib = _lib()
        abi.check(lib, lib.mgpu_fields_upload(self.h, dptr(u), dptr(p), dptr(flux), dptr(u_old), dptr(u_old_old)),
                  "mgpu_fields_upload")

    def upload_T(self, T, T_old=None, T_old_old=None):
        """fields_t%T (and its history; None: = T) for a case with ctrl.energy
        (mgpu_temperature_upload)."""
        conv = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        lib = _lib()
        abi.check(lib, lib.mgpu_temperature_upload(self.h, dptr(conv(T)), dptr(conv(T_old)), dptr(conv(T_old_old))),
                  "mgpu_temperature_upload")

    def temperature(self):
        """(T (N), gt (N, 3)): the temperature and its last Green-Gauss gradient."""
        T, gt = np.zeros(self.N), np.zeros((self.N, 3))
        lib = _lib()
        abi.check(lib, lib.mgpu_temperature_download(self.h, dptr(T), dptr(gt)), "mgpu_temperature_download")
        return T, gt

    FIELD_SHAPES = {"u": ("N", 3), "p": ("N",), "flux": ("F",), "gp": ("N", 3), "gu": ("N", 3, 3), "apc": ("N",)}

    def _field_arrays(self, out):
        N, F = self.N, self.F
        dims = {"N": N, "F": F}
        if out is None:
            return {k: np.empty(tuple(dims.get(d, d) for d in shp)) for k, shp in self.FIELD_SHAPES.items()}
        arrs = {}
        for k, a in out.items():
            want = tuple(dims.get(d, d) for d in self.FIELD_SHAPES[k])
            if a.dtype != np.float64 or a.shape != want or not a.flags.c_contiguous:
                raise ValueError(f"fields(out): {k} must be C-contiguous float64 of shape {want}")
            arrs[k] = a
        return arrs

    def simple_run_fields(self, nsteps: int = 0, out=None, logcap: int = 4096):
        """simple_run then fields(out) in one call (mgpu_simple_run_fields): the
        same results, the gp, gu and apc copies overlapping the last
        iteration's pressure solve when their arrays are page-locked. Returns
        (ier, records, fields) with fields as fields() returns them."""
        arrs = self._field_arrays(out)
        g = lambda k: dptr(arrs[k]) if k in arrs else None
        recs = (MgpuIterRec * max(logcap, 1))()
        nrec, ier = C.c_int(0), C.c_int(0)
        lib = _lib()
        abi.check(lib, lib.mgpu_simple_run_fields(self.h, int(nsteps), recs, int(logcap), C.byref(nrec),
                                                  C.byref(ier), g("u"), g("p"), g("flux"), g("gp"), g("gu"),
                                                  g("apc")), "mgpu_simple_run_fields")
        res = dict(arrs)
        if "gu" in res:
            res["gu"] = res["gu"].transpose(0, 2, 1)
        return ier.value, records_to_list(recs, min(nrec.value, logcap)), res

    def fields(self, out=None):
        """Host copies of u (N,3), p (N), flux (F), gp (N,3), gu (N,3,3) indexed
        [cell, component, direction] and apc (N).

        out: optional dict of caller-owned float64 C-contiguous arrays with some of
        those keys, filled in place (page-locked arrays copy fastest); only those
        fields are read back. Its "gu" array receives the C-ABI's layout
        gu(component, direction, cell), i.e. [cell, direction, component]; the
        returned "gu" is its transposed view."""
        arrs = self._field_arrays(out)
        g = lambda k: dptr(arrs[k]) if k in arrs else None
        lib = _lib()
        abi.check(lib, lib.mgpu_fields_download(self.h, g("u"), g("p"), g("flux"), g("gp"), g("gu"), g("apc")),
                  "mgpu_fields_download")
        res = dict(arrs)
        if "gu" in res:
            res["gu"] = res["gu"].transpose(0, 2, 1)
        return res

    def _run(self, fn, nsteps, logcap):
        recs = (MgpuIterRec * max(logcap, 1))()
        nrec, ier = C.c_int(0), C.c_int(0)
        lib = _lib()
        abi.check(lib, fn(self.h, int(nsteps), recs, int(logcap), C.byref(nrec), C.byref(ier)), fn.__name__)
        return ier.value, records_to_list(recs, min(nrec.value, logcap))

    def simple_run(self, nsteps: int = 0, logcap: int = 4096):
        """Steady SIMPLE; returns (ier, per-iteration records)."""
        return self._run(_lib().mgpu_simple_run, nsteps, logcap)

    def piso_run(self, nsteps: int = 0, logcap: int = 4096):
        """Transient PISO; returns (ier, per-step records)."""
        return self._run(_lib().mgpu_piso_run, nsteps, logcap)

    def pimple_run(self, nsteps: int = 0, logcap: int = 4096):
        """Transient PIMPLE (ctrl.n_outer_iter outer iterations per step); returns
        (ier, per-step records)."""
        return self._run(_lib().mgpu_pimple_run, nsteps, logcap)

    # ---- coupled mode (mod_uns_bc.f90:730-813, mod_uns_driver.f90:274-330) ----
    def interface_set(self, faces, u=None, p=None):
        """set_interface_vel / set_interface_p: faces 1-based, u (n, 3), p (n)."""
        faces = np.ascontiguousarray(faces, np.int32)
        u = None if u is None else np.ascontiguousarray(u, np.float64)
        p = None if p is None else np.ascontiguousarray(p, np.float64)
        lib = _lib()
        abi.check(lib, lib.mgpu_interface_set(self.h, len(faces), iptr(faces), dptr(u), dptr(p)),
                  "mgpu_interface_set")

    def interface_mode(self, p_dirichlet: bool):
        """set_iface_p_dirichlet: True when the peer supplies the face pressure."""
        lib = _lib()
        abi.check(lib, lib.mgpu_interface_mode(self.h, 1 if p_dirichlet else 0), "mgpu_interface_mode")

    def interface_set_T(self, faces, T=None, q=None, mode=None):
        """set_interface_T / set_interface_q / set_interface_T_mode (energy
        cases): faces 1-based; the peer's face temperature, heat flux into the
        domain and per-face mode (0 Dirichlet, 1 Neumann)."""
        faces = np.ascontiguousarray(faces, np.int32)
        T = None if T is None else np.ascontiguousarray(T, np.float64)
        q = None if q is None else np.ascontiguousarray(q, np.float64)
        mode = None if mode is None else np.ascontiguousarray(mode, np.int32)
        lib = _lib()
        abi.check(lib, lib.mgpu_interface_set_T(self.h, len(faces), iptr(faces), dptr(T), dptr(q), iptr(mode)),
                  "mgpu_interface_set_T")

    def interface_extract(self, with_T=False):
        """uns_solver_extract_iface for fluid owner cells: (faces 1-based, u (n, 3), p (n)),
        and T (n) with ``with_T``."""
        lib = _lib()
        n = C.c_int(0)
        abi.check(lib, lib.mgpu_interface_extract(self.h, 0, None, None, None, None, C.byref(n)),
                  "mgpu_interface_extract")
        faces = np.zeros(n.value, np.int32)
        u = np.zeros((n.value, 3))
        p = np.zeros(n.value)
        T = np.zeros(n.value)
        abi.check(lib, lib.mgpu_interface_extract(self.h, n.value, iptr(faces), dptr(u), dptr(p), dptr(T),
                                                  C.byref(n)), "mgpu_interface_extract")
        return (faces, u, p, T) if with_T else (faces, u, p)

    def nan_scan(self):
        """(ifin, field, cell, value, kind) of the first non-finite value."""
        ifin, field, cell, kind = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        val = C.c_double()
        lib = _lib()
        abi.check(lib, lib.mgpu_nan_scan(self.h, C.byref(ifin), C.byref(field), C.byref(cell), C.byref(val),
                                         C.byref(kind)), "mgpu_nan_scan")
        return ifin.value, field.value, cell.value, val.value, kind.value

    def stage(self, what: int, ts_order: int = 0, apc=None, nnz: int = 0, pp=None):
        """Run one kernel stage (see mgpu_case_stage); returns (aval, rhs, ap)."""
        lib = _lib()
        aval = np.zeros(max(nnz, 1)); rhs = np.zeros(self.N); ap = np.zeros(self.N)
        a = None if apc is None else np.ascontiguousarray(apc, np.float64)
        q = None if pp is None else np.ascontiguousarray(pp, np.float64)
        abi.check(lib, lib.mgpu_case_stage(self.h, int(what), int(ts_order), dptr(a), dptr(aval) if nnz else None,
                                           dptr(rhs), dptr(ap), dptr(q)), "mgpu_case_stage")
        return aval, rhs, ap

    def set_profiling(self, on: bool):
        _lib().mgpu_case_set_profiling(self.h, 1 if on else 0)

    def timing(self) -> dict:
        t = MgpuTiming()
        _lib().mgpu_case_timing(self.h, C.byref(t))
        return dict(total_ms=t.total_ms, krylov_launches=t.krylov_launches, krylov_ms=t.krylov_ms,
                    gpu_launches=t.gpu_launches)

    def solve_times(self) -> np.ndarray:
        """Device ms of each Krylov solve of the last profiled run, launch order."""
        lib = _lib()
        n = C.c_int(0)
        lib.mgpu_case_solve_times(self.h, None, 0, C.byref(n))
        out = np.zeros(max(n.value, 1))
        lib.mgpu_case_solve_times(self.h, dptr(out), n.value, C.byref(n))
        return out[:n.value]

    def device_bytes(self) -> int:
        b = C.c_int64()
        _lib().mgpu_case_device_bytes(self.h, C.byref(b))
        return int(b.value)

    def begin(self, mode: int, nsteps: int = 0) -> int:
        """Start a run (0 SIMPLE, 1 PISO) that a :class:`CaseBatch` steps;
        returns ier (30 / 31 for a PISO run the control rejects)."""
        ier = C.c_int(0)
        lib = _lib()
        abi.check(lib, lib.mgpu_case_begin(self.h, int(mode), int(nsteps), C.byref(ier)), "mgpu_case_begin")
        return ier.value

    def finish(self, logcap: int = 4096):
        """(ier, records) of a run begun by :meth:`begin`, as simple_run / piso_run return them."""
        recs = (MgpuIterRec * max(logcap, 1))()
        nrec, ier = C.c_int(0), C.c_int(0)
        lib = _lib()
        abi.check(lib, lib.mgpu_case_finish(self.h, recs, int(logcap), C.byref(nrec), C.byref(ier)),
                  "mgpu_case_finish")
        return ier.value, records_to_list(recs, min(nrec.value, logcap))


def batch_plan(rows, split_rows: int, wide_lanes: int, capacity: int, passes=None):
    """Lane plan of a batched Krylov phase (host only): per system its class
    (0 wide lanes, 1 single-block lanes) and the widths of the lanes."""
    r = np.ascontiguousarray(rows, np.int32)
    p = None if passes is None else np.ascontiguousarray(passes, np.float64)
    cls = np.zeros(len(r), np.int32)
    widths = np.zeros(max(int(capacity), 1), np.int32)
    nl = C.c_int(0)
    lib = _lib()
    abi.check(lib, lib.mgpu_batch_plan(len(r), iptr(r), dptr(p), int(split_rows), int(wide_lanes), int(capacity),
                                       iptr(cls), iptr(widths), C.byref(nl)), "mgpu_batch_plan")
    return cls, widths[:nl.value].copy()


class CaseBatch:
    """Resident cases advanced together (see mgpu_batch_* in include/mixgpu.h)."""

    def __init__(self, cases, policy=None):
        lib = _lib()
        self.cases = list(cases)
        arr = (C.c_void_p * len(self.cases))(*[c.h.value for c in self.cases])
        self.h = C.c_void_p()
        abi.check(lib, lib.mgpu_batch_create(arr, len(self.cases), C.byref(self.h)), "mgpu_batch_create")
        if policy is not None:
            self.set_policy(*policy)

    def close(self):
        if self.h:
            _lib().mgpu_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_policy(self, split_rows: int, wide_lanes: int):
        """Fixed lane policy (row threshold, wide lanes); (0, 0) = autotune."""
        lib = _lib()
        abi.check(lib, lib.mgpu_batch_set_policy(self.h, int(split_rows), int(wide_lanes)), "mgpu_batch_set_policy")

    def step(self, iters: int) -> int:
        """Advance every running member; returns how many still run."""
        active = C.c_int(0)
        lib = _lib()
        abi.check(lib, lib.mgpu_batch_step(self.h, int(iters), C.byref(active)), "mgpu_batch_step")
        return active.value

    def poll(self) -> np.ndarray:
        done = np.zeros(len(self.cases), np.int32)
        lib = _lib()
        abi.check(lib, lib.mgpu_batch_poll(self.h, iptr(done)), "mgpu_batch_poll")
        return done

    def run(self, modes, nsteps: int = 0):
        """begin + step to the end + finish; returns (nrec, ier) arrays."""
        K = len(self.cases)
        m = np.ascontiguousarray(np.broadcast_to(np.asarray(modes, np.int32), (K,)))
        nrec = np.zeros(K, np.int32)
        ier = np.zeros(K, np.int32)
        lib = _lib()
        abi.check(lib, lib.mgpu_batch_run(self.h, iptr(m), int(nsteps), iptr(nrec), iptr(ier)), "mgpu_batch_run")
        return nrec, ier

    def set_profiling(self, on: bool):
        _lib().mgpu_batch_set_profiling(self.h, 1 if on else 0)

    def info(self) -> dict:
        i = MgpuBatchInfo()
        _lib().mgpu_batch_info(self.h, C.byref(i))
        out = {k: getattr(i, k) for k, _ in MgpuBatchInfo._fields_}
        out["phase_ms"] = list(i.phase_ms)
        return out


def set_tuning(key: str, value: int) -> None:
    """Process-wide launch tunables (see mgpu_set_tuning)."""
    lib = _lib()
    abi.check(lib, lib.mgpu_set_tuning(key.encode(), int(value)), "mgpu_set_tuning")


def get_tuning(key: str) -> int:
    """The value in effect of a tuning key (mgpu_get_tuning)."""
    lib = _lib()
    v = C.c_int(0)
    abi.check(lib, lib.mgpu_get_tuning(key.encode(), C.byref(v)), "mgpu_get_tuning")
    return int(v.value)


def _krylov(method, row_ptr, col_idx, val, b, x, tol, maxit, norm_mode=0):
    lib = _lib()
    n = len(row_ptr) - 1
    rp = np.ascontiguousarray(row_ptr, np.int32); ci = np.ascontiguousarray(col_idx, np.int32)
    v = np.ascontiguousarray(val, np.float64); bb = np.ascontiguousarray(b, np.float64)
    xx = np.ascontiguousarray(x, np.float64).copy()
    it, ierr, res = C.c_int(), C.c_int(), C.c_double()
    abi.check(lib, lib.mgpu_krylov_solve(n, iptr(rp), iptr(ci), dptr(v), dptr(bb), dptr(xx), float(tol),
                                         int(maxit), int(method), int(norm_mode), C.byref(it), C.byref(res),
                                         C.byref(ierr)), "mgpu_krylov_solve")
    return xx, it.value, res.value, ierr.value


def bicgstab_ilu0(row_ptr, col_idx, val, b, x, tol, maxit, norm_mode=0):
    """bicgstab_ilu0 (mod_uns_linsolver.f90:148-224); 1-based CSR."""
    return _krylov(abi.KRY_BICGSTAB_ILU0, row_ptr, col_idx, val, b, x, tol, maxit, norm_mode)


def cg_jacobi(row_ptr, col_idx, val, b, x, tol, maxit, norm_mode=0):
    """cg_jacobi (mod_uns_linsolver.f90:230-291)."""
    return _krylov(abi.KRY_CG_JACOBI, row_ptr, col_idx, val, b, x, tol, maxit, norm_mode)


def cg_ic0(row_ptr, col_idx, val, b, x, tol, maxit, norm_mode=0):
    """cg_ic0 (mod_uns_linsolver.f90:405-461)."""
    return _krylov(abi.KRY_CG_IC0, row_ptr, col_idx, val, b, x, tol, maxit, norm_mode)


def bicgstab_jacobi(row_ptr, col_idx, val, b, x, tol, maxit, norm_mode=0):
    """BiCGStab with z = r/diag in place of ilu0_apply (no reference counterpart)."""
    return _krylov(abi.KRY_BICGSTAB_JACOBI, row_ptr, col_idx, val, b, x, tol, maxit, norm_mode)


def cg_ilu0(row_ptr, col_idx, val, b, x, tol, maxit, norm_mode=0):
    """PCG with ILU(0) as preconditioner (no reference counterpart)."""
    return _krylov(abi.KRY_CG_ILU0, row_ptr, col_idx, val, b, x, tol, maxit, norm_mode)


def pcg_poly(row_ptr, col_idx, val, b, x, tol, maxit, precision=abi.PREC_MIXED, cheb_degree=0):
    """The mixed-precision (or FP64 polynomial) pressure solver on a 1-based
    CSR system: Chebyshev-Jacobi PCG with reliable updates
    (mgpu_pcg_poly_solve). Returns (x, it, res, ierr) like cg_ic0."""
    lib = _lib()
    rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
    ci = np.ascontiguousarray(col_idx, dtype=np.int32)
    v = np.ascontiguousarray(val, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    xx = np.array(x, dtype=np.float64, copy=True)
    n = len(rp) - 1
    it, ierr, res = C.c_int(0), C.c_int(0), C.c_double(0.0)
    abi.check(lib, lib.mgpu_pcg_poly_solve(n, iptr(rp), iptr(ci), dptr(v), dptr(bb), dptr(xx), float(tol), int(maxit),
                                           int(precision), int(cheb_degree), C.byref(it), C.byref(res),
                                           C.byref(ierr)), "mgpu_pcg_poly_solve")
    return xx, it.value, res.value, ierr.value


def csr_matvec(row_ptr, col_idx, val, x):
    """csr_matvec (mod_uns_linsolver.f90:40-52)."""
    lib = _lib()
    n = len(row_ptr) - 1
    y = np.zeros(n)
    rp = np.ascontiguousarray(row_ptr, np.int32); ci = np.ascontiguousarray(col_idx, np.int32)
    abi.check(lib, lib.mgpu_csr_matvec(n, iptr(rp), iptr(ci), dptr(np.ascontiguousarray(val, np.float64)),
                                       dptr(np.ascontiguousarray(x, np.float64)), dptr(y)), "mgpu_csr_matvec")
    return y


def read_cas(path: str):
    """A Fluent ASCII .cas mesh read by the library (mgpu_cas_read, the record
    handling of read_cas in mod_uns_cas_reader.f90:44-523) as a FaceMesh.
    Raises ValueError with the reader's ier on a file it rejects."""
    from .meshgen import FaceMesh
    lib = _lib()
    m = abi.MgpuMesh()
    holder = C.c_void_p()
    ier = C.c_int(0)
    abi.check(lib, lib.mgpu_cas_read(str(path).encode(), C.byref(m), C.byref(holder), C.byref(ier)),
              "mgpu_cas_read")
    if ier.value != 0:
        raise ValueError(f"mgpu_cas_read: {path}: ier {ier.value}")
    try:
        nn, nf = m.nnodes, m.nfaces
        x = np.ctypeslib.as_array(m.x, shape=(3 * nn,)).reshape(nn, 3).copy()
        ptr = np.ctypeslib.as_array(m.fnode_ptr, shape=(nf + 1,)).copy()
        fnodes = np.ctypeslib.as_array(m.fnodes, shape=(int(ptr[-1]),)).copy()
        c0 = np.ctypeslib.as_array(m.c0, shape=(nf,)).copy()
        c1 = np.ctypeslib.as_array(m.c1, shape=(nf,)).copy()
        zone = np.ctypeslib.as_array(m.zone, shape=(nf,)).copy()
        n = C.c_int(0)
        lib.mgpu_cas_zone_names(holder, None, 0, C.byref(n))
        buf = C.create_string_buffer(n.value + 1)
        lib.mgpu_cas_zone_names(holder, buf, n.value + 1, C.byref(n))
        names = {}
        for line in buf.value.decode().splitlines():
            zid, name = line.split(" ", 1)
            names[int(zid)] = name
    finally:
        lib.mgpu_cas_free(holder)
    return FaceMesh(x, ptr.astype(np.int32), fnodes.astype(np.int32), c0.astype(np.int32), c1.astype(np.int32),
                    zone.astype(np.int32), int(m.ncells), names)


def build_connectivity(mesh) -> dict:
    """build_connectivity + build_cell_csr (1-based arrays)."""
    lib = _lib()
    arr = MeshArrays(mesh)
    N, F = mesh.ncells, mesh.nfaces
    nint = mesh.n_interior()
    cf_ptr = np.zeros(N + 1, np.int32); cf = np.zeros(2 * nint + (F - nint), np.int32)
    c2c_ptr = np.zeros(N + 1, np.int32); c2c = np.zeros(2 * nint, np.int32)
    row_ptr = np.zeros(N + 1, np.int32); col = np.zeros(N + 2 * nint, np.int32)
    nnz = C.c_int32(0)
    abi.check(lib, lib.mgpu_build_connectivity(C.byref(arr.struct), iptr(cf_ptr), iptr(cf), iptr(c2c_ptr),
                                               iptr(c2c), iptr(row_ptr), iptr(col), C.byref(nnz)),
              "mgpu_build_connectivity")
    return dict(cf_ptr=cf_ptr, cf=cf, c2c_ptr=c2c_ptr, c2c=c2c, row_ptr=row_ptr, col_idx=col[:nnz.value].copy())


def compute_geometry(mesh) -> dict:
    """compute_geometry + lf weights, computed on the device."""
    lib = _lib()
    arr = MeshArrays(mesh)
    N, F = mesh.ncells, mesh.nfaces
    xf = np.zeros((F, 3)); sf = np.zeros((F, 3)); area = np.zeros(F)
    vol = np.zeros(N); xc = np.zeros((N, 3)); lf = np.zeros(F)
    abi.check(lib, lib.mgpu_geometry(C.byref(arr.struct), dptr(xf), dptr(sf), dptr(area), dptr(vol), dptr(xc),
                                     dptr(lf)), "mgpu_geometry")
    return dict(xf=xf, sf=sf, area=area, vol=vol, xc=xc, lf=lf)


def rcm_order(mesh) -> np.ndarray:
    """Reverse Cuthill-McKee cell numbering: new_of_old (1-based)."""
    lib = _lib()
    arr = MeshArrays(mesh)
    out = np.zeros(mesh.ncells, np.int32)
    abi.check(lib, lib.mgpu_rcm_order(C.byref(arr.struct), iptr(out)), "mgpu_rcm_order")
    return out


def rcm_order_device(mesh) -> np.ndarray:
    """The same reverse Cuthill-McKee numbering computed on the GPU (new_of_old,
    1-based; equal to :func:`rcm_order` entry for entry)."""
    lib = _lib()
    arr = MeshArrays(mesh)
    out = np.zeros(mesh.ncells, np.int32)
    abi.check(lib, lib.mgpu_rcm_order_device(C.byref(arr.struct), iptr(out)), "mgpu_rcm_order_device")
    return out


def mesh_topology(mesh, on_device: bool = True) -> dict:
    """The integer arrays a case builds from its mesh (0-based): cell->face
    lists, CSR pattern, diagonal positions, face->slot map, transpose map and
    the triangular level sets; on the GPU (the path mgpu_case_create takes) or
    by the host builder."""
    lib = _lib()
    arr = MeshArrays(mesh)
    n = mesh.ncells
    sizes = np.zeros(4, np.int32)
    none = [None] * 11
    abi.check(lib, lib.mgpu_mesh_topology(C.byref(arr.struct), int(on_device), iptr(sizes), *none),
              "mgpu_mesh_topology")
    ncf, nnz, nlo, nup = (int(v) for v in sizes)
    out = {k: np.zeros(m, np.int32) for k, m in (("cf_ptr", n + 1), ("cf", ncf), ("row_ptr", n + 1), ("col", nnz),
                                                  ("diag", n), ("cf_slot", ncf), ("lt_pos", nnz),
                                                  ("lo_ptr", nlo + 1), ("lo_rows", n), ("up_ptr", nup + 1),
                                                  ("up_rows", n))}
    keys = ["cf_ptr", "cf", "row_ptr", "col", "diag", "cf_slot", "lt_pos", "lo_ptr", "lo_rows", "up_ptr", "up_rows"]
    abi.check(lib, lib.mgpu_mesh_topology(C.byref(arr.struct), int(on_device), iptr(sizes),
                                          *[iptr(out[k]) for k in keys]), "mgpu_mesh_topology")
    return out
