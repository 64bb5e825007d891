"""ctypes front end of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py, always as the checker or the timed
CPU baseline, never as part of the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from mixsolver_b200.abi import (MeshArrays, MgpuCtrl, MgpuIterRec, MgpuMesh, dptr, iptr,
                                records_to_list)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "oracle.cpp")):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        P = C.POINTER
        dp, ip = P(C.c_double), P(C.c_int32)
        L.orc_case_create.argtypes = [P(MgpuMesh), P(MgpuCtrl), P(C.c_void_p), P(C.c_int)]
        L.orc_case_destroy.argtypes = [C.c_void_p]
        L.orc_fields_upload.argtypes = [C.c_void_p, dp, dp, dp, dp, dp]
        L.orc_fields_download.argtypes = [C.c_void_p, dp, dp, dp, dp, dp, dp]
        L.orc_temperature_upload.argtypes = [C.c_void_p, dp, dp, dp]
        L.orc_temperature_download.argtypes = [C.c_void_p, dp, dp]
        L.orc_simple_run.argtypes = [C.c_void_p, C.c_int, P(MgpuIterRec), C.c_int, P(C.c_int), P(C.c_int)]
        L.orc_piso_run.argtypes = [C.c_void_p, C.c_int, P(MgpuIterRec), C.c_int, P(C.c_int), P(C.c_int)]
        L.orc_pimple_run.argtypes = [C.c_void_p, C.c_int, P(MgpuIterRec), C.c_int, P(C.c_int), P(C.c_int)]
        L.orc_geometry.argtypes = [C.c_void_p, dp, dp, dp, dp, dp, dp]
        L.orc_connectivity.argtypes = [C.c_void_p, ip, ip, ip, ip, ip, ip, ip]
        L.orc_stage.argtypes = [C.c_void_p, C.c_int, dp, dp, dp, dp]
        L.orc_set_apc.argtypes = [C.c_void_p, dp, C.c_int]
        L.orc_nan_scan.argtypes = [C.c_void_p, P(C.c_int), P(C.c_int), P(C.c_int), dp, P(C.c_int)]
        L.orc_interface_set.argtypes = [C.c_void_p, C.c_int, ip, dp, dp]
        L.orc_interface_mode.argtypes = [C.c_void_p, C.c_int]
        L.orc_interface_set_T.argtypes = [C.c_void_p, C.c_int, ip, dp, dp, ip]
        L.orc_interface_extract.argtypes = [C.c_void_p, C.c_int, ip, dp, dp, dp, P(C.c_int)]
        L.orc_krylov_solve.argtypes = [C.c_int, ip, ip, dp, dp, dp, C.c_double, C.c_int, C.c_int,
                                       C.c_int, P(C.c_int), dp, P(C.c_int)]
        L.orc_csr_matvec.argtypes = [C.c_int, ip, ip, dp, dp, dp]
        L.orc_factor.argtypes = [C.c_int, ip, ip, dp, C.c_int]
        L.orc_norm2.argtypes = [dp, C.c_long]
        L.orc_norm2.restype = C.c_double
        _lib = L
    return _lib


class OracleCase:
    """One mesh + control on the CPU oracle."""

    def __init__(self, mesh, ctrl):
        self.mesh = mesh
        self._arrays = MeshArrays(mesh)
        self._ctrl = ctrl.to_c()
        self.h = C.c_void_p()
        ier = C.c_int(0)
        rc = lib().orc_case_create(C.byref(self._arrays.struct), C.byref(self._ctrl), C.byref(self.h), C.byref(ier))
        if rc != 0:
            raise RuntimeError(f"oracle case_create failed rc={rc} ier={ier.value}")
        self.N, self.F = mesh.ncells, mesh.nfaces

    def close(self):
        if self.h:
            lib().orc_case_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, u=None, p=None, flux=None, u_old=None, u_old_old=None):
        conv = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        u, p, flux, u_old, u_old_old = map(conv, (u, p, flux, u_old, u_old_old))
        lib().orc_fields_upload(self.h, dptr(u), dptr(p), dptr(flux), dptr(u_old), dptr(u_old_old))

    def fields(self):
        u = np.zeros((self.N, 3)); p = np.zeros(self.N); flux = np.zeros(self.F)
        gp = np.zeros((self.N, 3)); gu = np.zeros((self.N, 3, 3)); apc = np.zeros(self.N)
        lib().orc_fields_download(self.h, dptr(u), dptr(p), dptr(flux), dptr(gp), dptr(gu), dptr(apc))
        # gu(comp,dir,cell) column-major == [cell][dir][comp] row-major
        return dict(u=u, p=p, flux=flux, gp=gp, gu=gu.transpose(0, 2, 1).copy(), apc=apc)

    def upload_T(self, T, T_old=None, T_old_old=None):
        conv = lambda a: None if a is None else np.ascontiguousarray(a, np.float64)
        lib().orc_temperature_upload(self.h, dptr(conv(T)), dptr(conv(T_old)), dptr(conv(T_old_old)))

    def temperature(self):
        T, gt = np.zeros(self.N), np.zeros((self.N, 3))
        lib().orc_temperature_download(self.h, dptr(T), dptr(gt))
        return T, gt

    def _run(self, fn, nsteps, logcap):
        recs = (MgpuIterRec * max(logcap, 1))()
        nrec, ier = C.c_int(0), C.c_int(0)
        fn(self.h, int(nsteps), recs, int(logcap), C.byref(nrec), C.byref(ier))
        return ier.value, records_to_list(recs, min(nrec.value, logcap))

    def simple_run(self, nsteps=0, logcap=4096):
        return self._run(lib().orc_simple_run, nsteps, logcap)

    def piso_run(self, nsteps=0, logcap=4096):
        return self._run(lib().orc_piso_run, nsteps, logcap)

    def pimple_run(self, nsteps=0, logcap=4096):
        return self._run(lib().orc_pimple_run, nsteps, logcap)

    def geometry(self):
        N, F = self.N, self.F
        xf = np.zeros((F, 3)); sf = np.zeros((F, 3)); area = np.zeros(F)
        vol = np.zeros(N); xc = np.zeros((N, 3)); lf = np.zeros(F)
        lib().orc_geometry(self.h, dptr(xf), dptr(sf), dptr(area), dptr(vol), dptr(xc), dptr(lf))
        return dict(xf=xf, sf=sf, area=area, vol=vol, xc=xc, lf=lf)

    def connectivity(self):
        N, F = self.N, self.F
        nint = self.mesh.n_interior()
        cf_ptr = np.zeros(N + 1, np.int32); cf = np.zeros(2 * nint + (F - nint), np.int32)
        c2c_ptr = np.zeros(N + 1, np.int32); c2c = np.zeros(2 * nint, np.int32)
        row_ptr = np.zeros(N + 1, np.int32); col = np.zeros(N + 2 * nint, np.int32)
        nnz = C.c_int32(0)
        lib().orc_connectivity(self.h, iptr(cf_ptr), iptr(cf), iptr(c2c_ptr), iptr(c2c), iptr(row_ptr),
                               iptr(col), C.byref(nnz))
        return dict(cf_ptr=cf_ptr, cf=cf, c2c_ptr=c2c_ptr, c2c=c2c, row_ptr=row_ptr,
                    col_idx=col[:nnz.value].copy())

    def stage(self, what, nnz=None, pp=None):
        aval = np.zeros(nnz if nnz else 1); rhs = np.zeros(self.N); ap = np.zeros(self.N)
        ppa = None if pp is None else np.ascontiguousarray(pp, np.float64)
        rc = lib().orc_stage(self.h, int(what), dptr(aval), dptr(rhs), dptr(ap), dptr(ppa))
        assert rc == 0
        return aval, rhs, ap

    def set_apc(self, apc=None, ts_order=0):
        a = None if apc is None else np.ascontiguousarray(apc, np.float64)
        lib().orc_set_apc(self.h, dptr(a), int(ts_order))

    def interface_set(self, faces, u=None, p=None):
        faces = np.ascontiguousarray(faces, np.int32)
        u = None if u is None else np.ascontiguousarray(u, np.float64)
        p = None if p is None else np.ascontiguousarray(p, np.float64)
        assert lib().orc_interface_set(self.h, len(faces), iptr(faces), dptr(u), dptr(p)) == 0

    def interface_set_T(self, faces, T=None, q=None, mode=None):
        faces = np.ascontiguousarray(faces, np.int32)
        T = None if T is None else np.ascontiguousarray(T, np.float64)
        q = None if q is None else np.ascontiguousarray(q, np.float64)
        mode = None if mode is None else np.ascontiguousarray(mode, np.int32)
        assert lib().orc_interface_set_T(self.h, len(faces), iptr(faces), dptr(T), dptr(q), iptr(mode)) == 0

    def interface_mode(self, p_dirichlet):
        lib().orc_interface_mode(self.h, 1 if p_dirichlet else 0)

    def interface_extract(self, with_T=False):
        n = C.c_int(0)
        lib().orc_interface_extract(self.h, 0, None, None, None, None, C.byref(n))
        faces, u, p, T = np.zeros(n.value, np.int32), np.zeros((n.value, 3)), np.zeros(n.value), np.zeros(n.value)
        lib().orc_interface_extract(self.h, n.value, iptr(faces), dptr(u), dptr(p), dptr(T), C.byref(n))
        return (faces, u, p, T) if with_T else (faces, u, p)

    def nan_scan(self):
        ifin, field, cell, kind = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        val = C.c_double()
        lib().orc_nan_scan(self.h, C.byref(ifin), C.byref(field), C.byref(cell), C.byref(val), C.byref(kind))
        return ifin.value, field.value, cell.value, val.value, kind.value


def krylov_solve(row_ptr, col_idx, val, b, x0, tol, maxit, method, norm_mode=0):
    """Stand-alone Krylov solve (1-based CSR); returns (x, it, res, ierr)."""
    n = len(row_ptr) - 1
    x = np.ascontiguousarray(x0, np.float64).copy()
    it, ierr, res = C.c_int(), C.c_int(), C.c_double()
    rp = np.ascontiguousarray(row_ptr, np.int32); ci = np.ascontiguousarray(col_idx, np.int32)
    v = np.ascontiguousarray(val, np.float64); bb = np.ascontiguousarray(b, np.float64)
    lib().orc_krylov_solve(n, iptr(rp), iptr(ci), dptr(v), dptr(bb), dptr(x), float(tol), int(maxit),
                           int(method), int(norm_mode), C.byref(it), C.byref(res), C.byref(ierr))
    return x, it.value, res.value, ierr.value


def csr_matvec(row_ptr, col_idx, val, x):
    n = len(row_ptr) - 1
    y = np.zeros(n)
    rp = np.ascontiguousarray(row_ptr, np.int32); ci = np.ascontiguousarray(col_idx, np.int32)
    lib().orc_csr_matvec(n, iptr(rp), iptr(ci), dptr(np.ascontiguousarray(val, np.float64)),
                         dptr(np.ascontiguousarray(x, np.float64)), dptr(y))
    return y


def factor(row_ptr, col_idx, val, kind):
    """kind 0 ILU(0) (ilu0_factor), 1 IC(0) (ic0_factor); returns (factored values, status)."""
    n = len(row_ptr) - 1
    v = np.ascontiguousarray(val, np.float64).copy()
    rp = np.ascontiguousarray(row_ptr, np.int32); ci = np.ascontiguousarray(col_idx, np.int32)
    e = lib().orc_factor(n, iptr(rp), iptr(ci), dptr(v), int(kind))
    return v, e


def norm2(a):
    a = np.ascontiguousarray(a, np.float64)
    return lib().orc_norm2(dptr(a), a.size)
