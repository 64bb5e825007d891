// oracle.cpp -- CPU FP64 restatement of MixSolver's unstructured SIMPLE/PISO
// pressure-velocity path. TEST INFRASTRUCTURE ONLY: it is the checker that the
// CUDA path is compared against (tests, the smoke check and the CPU-baseline
// leg of bench.py); nothing in the product links or calls it.
//
// Single-threaded and loop-order faithful: every loop visits faces/cells in the
// reference's order and every expression keeps the reference's association
// (Fortran evaluates a+b+c as (a+b)+c; -O2 gfortran on x86-64 issues no FMA),
// so this file must be compiled with -ffp-contract=off. Each function cites the
// Fortran routine it restates (paths relative to the reference project root).
//
// Pinning: the reference cannot be compiled here (no Fortran compiler). The
// restatement is pinned against the reference's published outputs: the Ghia
// centre-line L2 of the steady 80x80 and 40x40 cavities computed on the
// reference's own .cas meshes (cluster_cases/README.md:189-190,
// cluster_cases/cavity_Re1000/unMesh.control:63), and the NaN-guard semantics
// of src/unstructured/test_nan_guard.f90.
//
// Internal indices are 0-based (cell c <-> Fortran c+1); c1 < 0 marks a
// boundary face (Fortran c1 == 0).

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/mixgpu.h"

namespace {

using std::vector;
const double TINY = DBL_MIN;  // tiny(1.0_dp)

// gfortran's NORM2: the scaled sum of squares of the gfortran front end
// (scale starts at 1; a larger |x| rescales the running sum).
double norm2_scaled(const double* a, long n, long stride = 1) {
  double result = 0.0, scale = 1.0;
  for (long i = 0; i < n; ++i) {
    double v = a[i * stride];
    if (v != 0.0) {
      double ax = std::fabs(v);
      if (ax > scale) {
        double val = scale / ax;
        result = 1.0 + result * val * val;
        scale = ax;
      } else {
        double val = ax / scale;
        result += val * val;
      }
    }
  }
  return scale * std::sqrt(result);
}
inline double norm3(const double v[3]) { return norm2_scaled(v, 3); }
// dot_product of two 3-vectors as gfortran inlines it: ((0+a1b1)+a2b2)+a3b3
inline double dot3(const double* a, const double* b) {
  double s = 0.0;
  s = s + a[0] * b[0];
  s = s + a[1] * b[1];
  s = s + a[2] * b[2];
  return s;
}
double dotn(const double* a, const double* b, long n) {
  double s = 0.0;
  for (long i = 0; i < n; ++i) s = s + a[i] * b[i];
  return s;
}

// ---------------------------------------------------------------------------
// Mesh, connectivity, geometry
// ---------------------------------------------------------------------------
struct Mesh {
  int nnodes = 0, nfaces = 0, ncells = 0;
  vector<double> x;  // 3*nnodes
  vector<int> fptr, fnodes;  // fnodes 0-based
  vector<int> c0, c1, zone;  // c1 = -1 boundary
};

struct Conn {  // mod_uns_connectivity.f90:17-24 (0-based here)
  vector<int> cf_ptr, cf, c2c_ptr, c2c, bfaces;
};

// build_connectivity, mod_uns_connectivity.f90:28-108
void build_connectivity(const Mesh& m, Conn& c) {
  int n = m.ncells;
  c.cf_ptr.assign(n + 1, 0);
  for (int i = 0; i < m.nfaces; ++i) {
    c.cf_ptr[m.c0[i] + 1] += 1;
    if (m.c1[i] >= 0) c.cf_ptr[m.c1[i] + 1] += 1;
  }
  for (int k = 0; k < n; ++k) c.cf_ptr[k + 1] += c.cf_ptr[k];
  c.cf.assign(c.cf_ptr[n], 0);
  {
    vector<int> fill(c.cf_ptr.begin(), c.cf_ptr.end() - 1);
    for (int i = 0; i < m.nfaces; ++i) {
      int cell = m.c0[i];
      c.cf[fill[cell]++] = i;
      if (m.c1[i] >= 0) {
        cell = m.c1[i];
        c.cf[fill[cell]++] = i;
      }
    }
  }
  c.bfaces.clear();
  for (int i = 0; i < m.nfaces; ++i)
    if (m.c1[i] < 0) c.bfaces.push_back(i);
  c.c2c_ptr.assign(n + 1, 0);
  for (int i = 0; i < m.nfaces; ++i)
    if (m.c1[i] >= 0) {
      c.c2c_ptr[m.c0[i] + 1] += 1;
      c.c2c_ptr[m.c1[i] + 1] += 1;
    }
  for (int k = 0; k < n; ++k) c.c2c_ptr[k + 1] += c.c2c_ptr[k];
  c.c2c.assign(c.c2c_ptr[n], 0);
  {
    vector<int> fill(c.c2c_ptr.begin(), c.c2c_ptr.end() - 1);
    for (int i = 0; i < m.nfaces; ++i)
      if (m.c1[i] >= 0) {
        c.c2c[fill[m.c0[i]]++] = m.c1[i];
        c.c2c[fill[m.c1[i]]++] = m.c0[i];
      }
  }
}

struct Geom {  // geom_t, mod_uns_geometry.f90:22-30 (rc0/rc1 not used on the path)
  vector<double> xf, sf, area, vol, xc;
};

inline void cross(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// face_props, mod_uns_geometry.f90:97-131
void face_props(const Mesh& m, int i, double* cen, double* s, double& a) {
  int b = m.fptr[i], n = m.fptr[i + 1] - b;
  s[0] = s[1] = s[2] = 0.0;
  for (int j = 0; j < n; ++j) {
    int jn = (j + 1) % n;
    const double* p1 = &m.x[3 * m.fnodes[b + j]];
    const double* p2 = &m.x[3 * m.fnodes[b + jn]];
    double c[3];
    cross(p1, p2, c);
    for (int k = 0; k < 3; ++k) s[k] = s[k] + 0.5 * c[k];
  }
  a = norm3(s);
  cen[0] = cen[1] = cen[2] = 0.0;
  double at = 0.0;
  const double* p1 = &m.x[3 * m.fnodes[b]];
  for (int j = 1; j < n - 1; ++j) {
    const double* p2 = &m.x[3 * m.fnodes[b + j]];
    const double* p3 = &m.x[3 * m.fnodes[b + j + 1]];
    double u[3], v[3], st[3];
    for (int k = 0; k < 3; ++k) {
      u[k] = p2[k] - p1[k];
      v[k] = p3[k] - p1[k];
    }
    cross(u, v, st);
    for (int k = 0; k < 3; ++k) st[k] = st[k] * 0.5;
    double ns = norm3(st);
    for (int k = 0; k < 3; ++k) cen[k] = cen[k] + ns * ((p1[k] + p2[k]) + p3[k]) / 3.0;
    at = at + ns;
  }
  if (at > 0.0)
    for (int k = 0; k < 3; ++k) cen[k] = cen[k] / at;
}

// compute_geometry, mod_uns_geometry.f90:40-92 (prov_centers :134-158,
// accumulate_cell :161-174)
void compute_geometry(const Mesh& m, Geom& g) {
  int F = m.nfaces, N = m.ncells;
  g.xf.assign(3 * F, 0.0);
  g.sf.assign(3 * F, 0.0);
  g.area.assign(F, 0.0);
  g.vol.assign(N, 0.0);
  g.xc.assign(3 * N, 0.0);
  for (int i = 0; i < F; ++i) face_props(m, i, &g.xf[3 * i], &g.sf[3 * i], g.area[i]);
  vector<double> pcen(3 * N, 0.0);
  vector<int> cnt(N, 0);
  for (int i = 0; i < F; ++i) {
    int c0 = m.c0[i], c1 = m.c1[i];
    for (int j = m.fptr[i]; j < m.fptr[i + 1]; ++j) {
      const double* xn = &m.x[3 * m.fnodes[j]];
      for (int k = 0; k < 3; ++k) pcen[3 * c0 + k] = pcen[3 * c0 + k] + xn[k];
      cnt[c0] += 1;
      if (c1 >= 0) {
        for (int k = 0; k < 3; ++k) pcen[3 * c1 + k] = pcen[3 * c1 + k] + xn[k];
        cnt[c1] += 1;
      }
    }
  }
  for (int i = 0; i < N; ++i)
    if (cnt[i] > 0)
      for (int k = 0; k < 3; ++k) pcen[3 * i + k] = pcen[3 * i + k] / (double)cnt[i];
  for (int i = 0; i < F; ++i) {
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = g.xf[3 * i + k] - pcen[3 * m.c0[i] + k];
    double dotv = dot3(&g.sf[3 * i], d);
    if (dotv < 0.0)
      for (int k = 0; k < 3; ++k) g.sf[3 * i + k] = -g.sf[3 * i + k];
  }
  const double THIRD = 1.0 / 3.0, QRTR = 1.0 / 4.0;
  auto acc = [&](const double* p, int sgn, int i, int cell) {
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = g.xf[3 * i + k] - p[k];
    double dv = THIRD * dot3(&g.sf[3 * i], d) * (double)sgn;
    g.vol[cell] = g.vol[cell] + dv;
    for (int k = 0; k < 3; ++k)
      g.xc[3 * cell + k] = g.xc[3 * cell + k] + dv * ((1.0 - QRTR) * g.xf[3 * i + k] + QRTR * p[k]);
  };
  for (int i = 0; i < F; ++i) {
    acc(&pcen[3 * m.c0[i]], +1, i, m.c0[i]);
    if (m.c1[i] >= 0) acc(&pcen[3 * m.c1[i]], -1, i, m.c1[i]);
  }
  for (int k = 0; k < N; ++k)
    if (g.vol[k] > 0.0)
      for (int d = 0; d < 3; ++d) g.xc[3 * k + d] = g.xc[3 * k + d] / g.vol[k];
}

// ---------------------------------------------------------------------------
// Boundary conditions (mod_uns_bc.f90)
// ---------------------------------------------------------------------------
struct Group {
  int zone = 0, btype = 0;
  double uvel[3] = {0, 0, 0}, pval = 0, mdot = 0, uspeed = 0;
  double prfl_mean = 0, prfl_span = 1, prfl_origin = 0;
  int prfl_axis = 2;
  bool has_lid = false;
  int lid_dir = 0;
  double lid_coord = 0, lid_tol = 0, lid_vel[3] = {0, 0, 0};
  vector<int> faces;
  // thermal data (bc_group_t, mod_uns_bc.f90:95-105): zone-level type and
  // values, plane filters and their match tolerance
  int ttype = 0;
  double tval = 0, qval = 0;
  int ntbc = 0, tbc_pdir[4] = {0, 0, 0, 0}, tbc_ttype[4] = {0, 0, 0, 0};
  double tbc_pcoord[4] = {0, 0, 0, 0}, tbc_tval[4] = {0, 0, 0, 0}, tbc_qval[4] = {0, 0, 0, 0};
  double tbc_tol = 0;
};
struct BC {
  vector<Group> gb;
  vector<int> fgrp;  // face -> group index (0-based), -1 interior
  double inlet_ramp = 1.0, pval_ramp = 1.0;  // g_inlet_ramp_factor / g_pval_ramp_factor
  // coupling interface (mod_uns_bc.f90:117-130, 730-813): iface_vel(3,nfaces),
  // iface_p(nfaces), g_iface_p_dir
  vector<double> iface_vel, iface_p;
  bool iface_p_dir = false;
  // iface_T, iface_q, iface_T_mode (mod_uns_bc.f90:125-144): the peer's face
  // temperature, its heat flux into the domain, 0 Dirichlet / 1 Neumann
  vector<double> iface_T, iface_q;
  vector<int> iface_T_mode;
};

// build_bc, mod_uns_bc.f90:155-393 (interface zones are not part of this path)
int build_bc(const Mesh& m, const MgpuCtrl& ctrl, BC& bcs) {
  bcs.gb.assign(ctrl.nbc, Group());
  bcs.fgrp.assign(m.nfaces, -1);
  double cmax[3], cmin[3];
  for (int k = 0; k < 3; ++k) cmax[k] = -HUGE_VAL, cmin[k] = HUGE_VAL;
  for (int i = 0; i < m.nnodes; ++i)
    for (int k = 0; k < 3; ++k) {
      cmax[k] = std::max(cmax[k], m.x[3 * i + k]);
      cmin[k] = std::min(cmin[k], m.x[3 * i + k]);
    }
  double crange = 0.0;
  for (int k = 0; k < 3; ++k) crange = std::max(crange, cmax[k] - cmin[k]);
  for (int i = 0; i < ctrl.nbc; ++i) {
    const MgpuBcSpec& sp = ctrl.bc[i];
    Group& gb = bcs.gb[i];
    gb.zone = sp.zone;
    gb.btype = sp.btype;
    for (int k = 0; k < 3; ++k) gb.uvel[k] = sp.uvel[k];
    gb.pval = sp.pval;
    gb.mdot = sp.mdot;
    gb.prfl_mean = sp.umean;
    gb.prfl_span = sp.uspan;
    gb.prfl_origin = sp.uorigin;
    gb.prfl_axis = sp.uaxis;
    if (sp.btype == MGPU_BC_VINLET_PARAB &&
        (gb.prfl_span <= 0.0 || gb.prfl_axis < 1 || gb.prfl_axis > 3))
      return 14;
    if (sp.btype == MGPU_BC_MASSINLET) {
      if (ctrl.rho <= 0.0) return 13;
      gb.uspeed = sp.mdot / ctrl.rho;
    }
    gb.has_lid = sp.has_lid != 0;
    gb.lid_dir = sp.lid_dir;
    gb.lid_coord = sp.lid_coord;
    for (int k = 0; k < 3; ++k) gb.lid_vel[k] = sp.lid_vel[k];
    if (gb.has_lid) gb.lid_tol = 1.0e-4 * crange;
    gb.ttype = sp.ttype;
    gb.tval = sp.tval;
    gb.qval = sp.qval;
    // tbc_plane lines of this zone (parse_tbc_plane keeps at most 4, in order)
    for (int t = 0; t < ctrl.ntbc && t < MGPU_MAXTBC; ++t) {
      const MgpuTbcPlane& pl = ctrl.tbc[t];
      if (pl.bc != i) continue;
      if (gb.ntbc >= 4) return 15;
      gb.tbc_pdir[gb.ntbc] = pl.pdir;
      gb.tbc_pcoord[gb.ntbc] = pl.pcoord;
      gb.tbc_ttype[gb.ntbc] = pl.ttype;
      gb.tbc_tval[gb.ntbc] = pl.tval;
      gb.tbc_qval[gb.ntbc] = pl.qval;
      ++gb.ntbc;
    }
    if (gb.ntbc > 0) gb.tbc_tol = 1.0e-4 * crange;
    int nb = 0;
    bool zone_known = false;
    for (int k = 0; k < m.nfaces; ++k) {
      if (m.zone[k] == sp.zone) zone_known = true;
      if (m.c1[k] < 0 && m.zone[k] == sp.zone) ++nb;
    }
    if (!zone_known) return 10;
    if (nb == 0) return 11;
    for (int k = 0; k < m.nfaces; ++k)
      if (m.c1[k] < 0 && m.zone[k] == sp.zone) {
        gb.faces.push_back(k);
        bcs.fgrp[k] = i;
      }
  }
  for (int k = 0; k < m.nfaces; ++k)
    if (m.c1[k] < 0 && bcs.fgrp[k] < 0) return 12;
  return 0;
}

// bc_face_vel, mod_uns_bc.f90:400-509
void bc_face_vel(const BC& bcs, int i, const double* xf, const double* sf, const double* uP, double* uf) {
  const Group& g = bcs.gb[bcs.fgrp[i]];
  double nvec[3], un, xi, uspc, ns;
  switch (g.btype) {
    case MGPU_BC_INTERFACE:  // mod_uns_bc.f90:460-475
      if (bcs.iface_p_dir)
        for (int k = 0; k < 3; ++k) uf[k] = uP[k];
      else
        for (int k = 0; k < 3; ++k) uf[k] = bcs.iface_vel[3 * (size_t)i + k];
      break;
    case MGPU_BC_WALL:
      if (g.has_lid && std::fabs(xf[g.lid_dir - 1] - g.lid_coord) <= g.lid_tol)
        for (int k = 0; k < 3; ++k) uf[k] = g.lid_vel[k];
      else
        uf[0] = uf[1] = uf[2] = 0.0;
      break;
    case MGPU_BC_SYMMETRY:
      ns = norm3(sf);
      for (int k = 0; k < 3; ++k) nvec[k] = sf[k] / ns;
      un = dot3(uP, nvec);
      for (int k = 0; k < 3; ++k) uf[k] = uP[k] - 2.0 * un * nvec[k];
      break;
    case MGPU_BC_VINLET:
      for (int k = 0; k < 3; ++k) uf[k] = g.uvel[k];
      break;
    case MGPU_BC_VINLET_PARAB:
      ns = norm3(sf);
      for (int k = 0; k < 3; ++k) nvec[k] = sf[k] / ns;
      xi = (xf[g.prfl_axis - 1] - g.prfl_origin) / g.prfl_span;
      xi = std::max(0.0, std::min(1.0, xi));
      uspc = 6.0 * g.prfl_mean * xi * (1.0 - xi);
      for (int k = 0; k < 3; ++k) uf[k] = -uspc * nvec[k];
      break;
    case MGPU_BC_MASSINLET:
      ns = norm3(sf);
      for (int k = 0; k < 3; ++k) nvec[k] = sf[k] / ns;
      for (int k = 0; k < 3; ++k) uf[k] = -g.uspeed * bcs.inlet_ramp * nvec[k];
      break;
    case MGPU_BC_FARFIELD:
      ns = norm3(sf);
      for (int k = 0; k < 3; ++k) nvec[k] = sf[k] / ns;
      un = dot3(g.uvel, nvec);
      if (un < 0.0)
        for (int k = 0; k < 3; ++k) uf[k] = g.uvel[k];
      else
        for (int k = 0; k < 3; ++k) uf[k] = uP[k];
      break;
    case MGPU_BC_SLIPWALL:
      ns = norm3(sf);
      for (int k = 0; k < 3; ++k) nvec[k] = sf[k] / ns;
      un = dot3(uP, nvec);
      for (int k = 0; k < 3; ++k) uf[k] = uP[k] - un * nvec[k];
      break;
    default:  // POUTLET, OUTFLOW and anything else: zeroth-order extrapolation
      for (int k = 0; k < 3; ++k) uf[k] = uP[k];
  }
}

// bc_face_p, mod_uns_bc.f90:514-549
inline double bc_face_p(const BC& bcs, int i, double pP) {
  const Group& g = bcs.gb[bcs.fgrp[i]];
  if (g.btype == MGPU_BC_POUTLET || g.btype == MGPU_BC_FARFIELD) return g.pval * bcs.pval_ramp;
  if (g.btype == MGPU_BC_INTERFACE) return bcs.iface_p_dir ? bcs.iface_p[i] : pP;  // :527-544
  return pP;
}

// bc_face_p_dirichlet, mod_uns_bc.f90:879-893
inline bool bc_face_p_dirichlet(const BC& bcs, int i) {
  int g = bcs.fgrp[i];
  if (g < 0) return false;
  int bt = bcs.gb[g].btype;
  if (bt == MGPU_BC_INTERFACE) return bcs.iface_p_dir;
  return bt == MGPU_BC_POUTLET || bt == MGPU_BC_FARFIELD;
}

// the Dirichlet rule of the one-rank ppe_assembly_mpi (mod_uns_simple_mpi.f90:
// 905-907, 944-945), which the transient drivers use: pressure outlets and far
// fields only
inline bool ppe_dirichlet_mpi(const BC& bcs, int i) {
  int g = bcs.fgrp[i];
  if (g < 0) return false;
  int bt = bcs.gb[g].btype;
  return bt == MGPU_BC_POUTLET || bt == MGPU_BC_FARFIELD;
}

// bc_face_T, mod_uns_bc.f90:560-703 (without the porous/solid phase split):
// T_face, q_face and whether the face is Neumann. Interface faces take the
// peer's temperature (iface_T), or its heat flux in the CHT mode (:687-691).
void bc_face_T(const BC& bcs, int i, const double* xf, double T_cell, double& T_face, double& q_face,
               bool& is_neumann) {
  const Group& gb = bcs.gb[bcs.fgrp[i]];
  T_face = T_cell;
  q_face = 0.0;
  is_neumann = true;
  auto typed = [&](bool wall) {
    int tt = gb.ttype;
    double tv = gb.tval, qv = gb.qval;
    for (int ipl = 0; ipl < gb.ntbc; ++ipl)
      if (std::fabs(xf[gb.tbc_pdir[ipl] - 1] - gb.tbc_pcoord[ipl]) <= gb.tbc_tol) {
        tt = gb.tbc_ttype[ipl];
        tv = gb.tbc_tval[ipl];
        qv = gb.tbc_qval[ipl];
        break;
      }
    if (tt == 1) {
      is_neumann = false;
      T_face = tv;
      q_face = 0.0;
    } else if (tt == 2) {
      is_neumann = true;
      q_face = qv;
      T_face = T_cell;
    } else if (wall || tt == 0) {
      is_neumann = true;
      q_face = 0.0;
      T_face = T_cell;
    }
  };
  switch (gb.btype) {
    case MGPU_BC_WALL:
      typed(true);
      break;
    case MGPU_BC_SYMMETRY:
    case MGPU_BC_FARFIELD:
      break;
    case MGPU_BC_VINLET:
    case MGPU_BC_VINLET_PARAB:
    case MGPU_BC_MASSINLET:
      is_neumann = false;
      T_face = gb.tval;
      q_face = 0.0;
      break;
    case MGPU_BC_POUTLET:
    case MGPU_BC_OUTFLOW:
      typed(false);
      break;
    case MGPU_BC_INTERFACE:
      if (bcs.iface_T_mode[i] == 1) {
        is_neumann = true;
        q_face = bcs.iface_q[i];
        T_face = T_cell;
        break;
      }
      is_neumann = false;
      q_face = 0.0;
      T_face = bcs.iface_T[i];
      break;
    default:
      break;
  }
}

// ---------------------------------------------------------------------------
// CSR and Krylov solvers (mod_uns_linsolver.f90, mod_uns_linsolver_mpi.f90)
// ---------------------------------------------------------------------------
struct CSR {  // csr_t, mod_uns_linsolver.f90:27-33 (0-based)
  int nrows = 0;
  vector<int> row_ptr, col_idx, diag_pos;
  vector<double> val;
};

// csr_matvec, mod_uns_linsolver.f90:40-52
void csr_matvec(const CSR& A, const double* x, double* y) {
  for (int i = 0; i < A.nrows; ++i) {
    y[i] = 0.0;
    for (int k = A.row_ptr[i]; k < A.row_ptr[i + 1]; ++k) y[i] = y[i] + A.val[k] * x[A.col_idx[k]];
  }
}

// csr_find, mod_uns_linsolver.f90:57-71 (-1 when absent)
int csr_find(const CSR& A, int i, int j) {
  for (int k = A.row_ptr[i]; k < A.row_ptr[i + 1]; ++k) {
    if (A.col_idx[k] == j) return k;
    if (A.col_idx[k] > j) return -1;
  }
  return -1;
}

// ilu0_factor, mod_uns_linsolver.f90:79-115
int ilu0_factor(CSR& A) {
  A.diag_pos.assign(A.nrows, -1);
  for (int i = 0; i < A.nrows; ++i) {
    A.diag_pos[i] = csr_find(A, i, i);
    if (A.diag_pos[i] < 0) return 1;
  }
  for (int i = 1; i < A.nrows; ++i) {
    for (int kk = A.row_ptr[i]; kk < A.diag_pos[i]; ++kk) {
      int k = A.col_idx[kk];
      if (std::fabs(A.val[A.diag_pos[k]]) < TINY) return 2;
      double aik = A.val[kk] / A.val[A.diag_pos[k]];
      A.val[kk] = aik;
      for (int jj = A.diag_pos[k]; jj < A.row_ptr[k + 1]; ++jj) {
        int j = A.col_idx[jj];
        if (j <= k) continue;
        int pos = csr_find(A, i, j);
        if (pos >= 0) A.val[pos] = A.val[pos] - aik * A.val[jj];
      }
    }
  }
  return 0;
}

// ilu0_apply, mod_uns_linsolver.f90:120-142
void ilu0_apply(const CSR& A, const double* r, double* z) {
  int n = A.nrows;
  for (int i = 0; i < n; ++i) z[i] = r[i];
  for (int i = 0; i < n; ++i) {
    double s = z[i];
    for (int k = A.row_ptr[i]; k < A.diag_pos[i]; ++k) s = s - A.val[k] * z[A.col_idx[k]];
    z[i] = s;
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = z[i];
    for (int k = A.diag_pos[i] + 1; k < A.row_ptr[i + 1]; ++k) s = s - A.val[k] * z[A.col_idx[k]];
    z[i] = s / A.val[A.diag_pos[i]];
  }
}

// ic0_dot, mod_uns_linsolver.f90:297-314 (inclusive index ranges)
double ic0_dot(const CSR& A, int p1, int p2, int q1, int q2) {
  int p = p1, q = q1;
  double s = 0.0;
  while (p <= p2 && q <= q2) {
    if (A.col_idx[p] < A.col_idx[q])
      ++p;
    else if (A.col_idx[p] > A.col_idx[q])
      ++q;
    else {
      s = s + A.val[p] * A.val[q];
      ++p;
      ++q;
    }
  }
  return s;
}

// ic0_factor, mod_uns_linsolver.f90:328-365
int ic0_factor(CSR& A) {
  A.diag_pos.assign(A.nrows, -1);
  for (int i = 0; i < A.nrows; ++i) {
    A.diag_pos[i] = csr_find(A, i, i);
    if (A.diag_pos[i] < 0) return 1;
  }
  for (int i = 0; i < A.nrows; ++i) {
    int dpi = A.diag_pos[i];
    for (int kp = A.row_ptr[i]; kp < dpi; ++kp) {
      int k = A.col_idx[kp];
      double s = A.val[kp] - ic0_dot(A, A.row_ptr[i], kp - 1, A.row_ptr[k], A.diag_pos[k] - 1);
      A.val[kp] = s / A.val[A.diag_pos[k]];
    }
    double s = A.val[dpi];
    for (int kp = A.row_ptr[i]; kp < dpi; ++kp) s = s - A.val[kp] * A.val[kp];
    if (s <= 0.0) return 2;
    A.val[dpi] = std::sqrt(s);
  }
  return 0;
}

// ic0_apply, mod_uns_linsolver.f90:371-399
void ic0_apply(const CSR& L, const double* r, double* z, vector<double>& w) {
  int n = L.nrows;
  for (int i = 0; i < n; ++i) {
    double s = r[i];
    for (int kp = L.row_ptr[i]; kp < L.diag_pos[i]; ++kp) s = s - L.val[kp] * z[L.col_idx[kp]];
    z[i] = s / L.val[L.diag_pos[i]];
  }
  w.assign(z, z + n);
  for (int i = n - 1; i >= 0; --i) {
    z[i] = w[i] / L.val[L.diag_pos[i]];
    for (int kp = L.row_ptr[i]; kp < L.diag_pos[i]; ++kp) {
      int k = L.col_idx[kp];
      w[k] = w[k] - L.val[kp] * z[i];
    }
  }
}

// Krylov norm: the serial solvers use gfortran NORM2; the distributed solvers
// of mod_uns_linsolver_mpi.f90 at one rank use sqrt(gdot(a,a)) (:40-49).
struct Norm {
  int mode;  // 0 serial, 1 mpi-at-one-rank
  double operator()(const double* a, long n) const {
    return mode == 0 ? norm2_scaled(a, n) : std::sqrt(dotn(a, a, n));
  }
};

struct Precond {
  int kind;  // 0 ILU0, 1 Jacobi, 2 IC0
  bool strict_diag;  // Jacobi: also reject |diag| < tiny (distributed solvers)
  CSR f;     // factor copy (ILU0/IC0)
  vector<double> diag;
  vector<double> w;
  int setup(const CSR& A) {
    if (kind == 0) {
      f = A;
      return ilu0_factor(f);
    }
    if (kind == 2) {
      f = A;
      return ic0_factor(f);
    }
    diag.assign(A.nrows, 0.0);
    for (int i = 0; i < A.nrows; ++i) {
      int k = csr_find(A, i, i);
      if (k < 0 || (strict_diag && std::fabs(A.val[k]) < TINY)) return 2;
      diag[i] = A.val[k];
    }
    return 0;
  }
  void apply(const double* r, double* z) {
    if (kind == 0)
      ilu0_apply(f, r, z);
    else if (kind == 2)
      ic0_apply(f, r, z, w);
    else
      for (int i = 0; i < (int)diag.size(); ++i) z[i] = r[i] / diag[i];
  }
};

// bicgstab_ilu0, mod_uns_linsolver.f90:148-224 (serial) and bicgstab_ilu0_mpi,
// mod_uns_linsolver_mpi.f90:155-229 (one rank); the Jacobi variant replaces
// ilu0_apply by z = r/diag (configuration-required extension).
void bicgstab(const CSR& A, const double* b, double* x, double tol, int maxit, int& it, double& res,
              int& ierr, int pkind, Norm nrm) {
  int n = A.nrows;
  it = 0;
  ierr = 0;
  res = 0.0;
  double bnrm = nrm(b, n);
  if (bnrm == 0.0) {
    for (int i = 0; i < n; ++i) x[i] = 0.0;
    return;
  }
  Precond M{pkind, true};
  int fe = M.setup(A);
  if (fe != 0) {
    ierr = fe + 10;
    return;
  }
  vector<double> r0(n), r(n), p(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n), tmp(n);
  csr_matvec(A, x, tmp.data());
  for (int i = 0; i < n; ++i) r0[i] = b[i] - tmp[i];
  r = r0;
  double rho_old = 1.0, alpha = 1.0, omega = 1.0, rho, beta, tt, snrm;
  res = nrm(r0.data(), n) / bnrm;
  if (res <= tol) return;
  for (it = 1; it <= maxit; ++it) {
    rho = dotn(r.data(), r0.data(), n);
    if (std::fabs(rho) < TINY) {
      ierr = 2;
      break;
    }
    beta = (rho / rho_old) * (alpha / omega);
    for (int i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
    M.apply(p.data(), ph.data());
    csr_matvec(A, ph.data(), v.data());
    alpha = rho / dotn(r0.data(), v.data(), n);
    for (int i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
    snrm = nrm(s.data(), n);
    if (snrm / bnrm <= tol) {
      for (int i = 0; i < n; ++i) x[i] = x[i] + alpha * ph[i];
      res = snrm / bnrm;
      return;
    }
    M.apply(s.data(), sh.data());
    csr_matvec(A, sh.data(), t.data());
    tt = dotn(t.data(), t.data(), n);
    if (tt < TINY) {
      ierr = 2;
      break;
    }
    omega = dotn(t.data(), s.data(), n) / tt;
    if (std::fabs(omega) < TINY) {
      ierr = 2;
      break;
    }
    for (int i = 0; i < n; ++i) x[i] = x[i] + alpha * ph[i] + omega * sh[i];
    for (int i = 0; i < n; ++i) r[i] = s[i] - omega * t[i];
    res = nrm(r.data(), n) / bnrm;
    if (res <= tol) return;
    rho_old = rho;
  }
  if (ierr == 0) {
    ierr = 1;
    it = maxit;
  }
}

// cg_jacobi (:230-291) / cg_ic0 (:405-461) and their one-rank distributed twins
// (mod_uns_linsolver_mpi.f90:235-363); pkind 1 Jacobi, 2 IC0, 0 ILU0
// (PCG+ILU(0), configuration-required extension). On reaching maxit the DO
// variable is left at maxit+1 (Fortran loop semantics), as in the reference.
void pcg(const CSR& A, const double* b, double* x, double tol, int maxit, int& it, double& res,
         int& ierr, int pkind, Norm nrm) {
  int n = A.nrows;
  it = 0;
  ierr = 0;
  res = 0.0;
  double bnrm = nrm(b, n);
  if (bnrm == 0.0) {
    for (int i = 0; i < n; ++i) x[i] = 0.0;
    return;
  }
  Precond M{pkind, nrm.mode == 1};
  int fe = M.setup(A);
  if (fe != 0) {
    // cg_jacobi: a missing diagonal is a breakdown (ierr = 2, :253-259);
    // cg_jacobi_mpi also rejects |diag| < tiny the same way (:260-271)
    ierr = (pkind == 1) ? 2 : fe + 10;
    return;
  }
  vector<double> r(n), z(n), p(n), ap(n);
  csr_matvec(A, x, ap.data());
  for (int i = 0; i < n; ++i) r[i] = b[i] - ap[i];
  res = nrm(r.data(), n) / bnrm;
  if (res <= tol) return;
  M.apply(r.data(), z.data());
  p = z;
  double rz = dotn(r.data(), z.data(), n), rz_new, pap, alpha, beta;
  for (it = 1; it <= maxit; ++it) {
    csr_matvec(A, p.data(), ap.data());
    pap = dotn(p.data(), ap.data(), n);
    if (std::fabs(pap) < TINY) {
      ierr = 2;
      break;
    }
    alpha = rz / pap;
    for (int i = 0; i < n; ++i) x[i] = x[i] + alpha * p[i];
    for (int i = 0; i < n; ++i) r[i] = r[i] - alpha * ap[i];
    res = nrm(r.data(), n) / bnrm;
    if (res <= tol) return;
    M.apply(r.data(), z.data());
    rz_new = dotn(r.data(), z.data(), n);
    if (std::fabs(rz) < TINY) {
      ierr = 2;
      break;
    }
    beta = rz_new / rz;
    for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    rz = rz_new;
  }
  if (ierr == 0) ierr = 1;
}

// ---------------------------------------------------------------------------
// The case: fields and the SIMPLE / PISO algorithms (mod_uns_simple.f90)
// ---------------------------------------------------------------------------
struct Case {
  Mesh m;
  Conn conn;
  Geom g;
  BC bcs;
  MgpuCtrl ctrl;
  CSR amat, pmat;
  // fields_t (mod_uns_fields.f90:29-79); u, gu cell-major like the Fortran arrays
  vector<double> u, p, gp, gu, flux, lf, apc, u_old, u_old_old;
  vector<double> T, T_old, T_old_old, gt;  // fields_t%T, T_old, T_old_old, gt (3 per cell)
  int ts_order = 0;
  bool pimple = false;  // ctrl%pimple: pimple_run sets it for its run
  vector<double> rhs, ap, pp, phif, dpp, psi;
};

// build_cell_csr + sort_int, mod_uns_simple.f90:835-904
void build_cell_csr(const Mesh& m, const Conn& conn, CSR& A) {
  A.nrows = m.ncells;
  A.row_ptr.assign(m.ncells + 1, 0);
  A.col_idx.clear();
  vector<int> tmp, row;
  for (int k = 0; k < m.ncells; ++k) {
    int n = conn.c2c_ptr[k + 1] - conn.c2c_ptr[k];
    tmp.assign(conn.c2c.begin() + conn.c2c_ptr[k], conn.c2c.begin() + conn.c2c_ptr[k + 1]);
    tmp.push_back(k);
    for (int i = 1; i < n + 1; ++i) {  // insertion sort, ascending
      int key = tmp[i], j = i - 1;
      while (j >= 0 && tmp[j] > key) {
        tmp[j + 1] = tmp[j];
        --j;
      }
      tmp[j + 1] = key;
    }
    row.clear();
    for (int j = 0; j < n + 1; ++j)
      if (row.empty() || tmp[j] != row.back()) row.push_back(tmp[j]);
    A.row_ptr[k + 1] = A.row_ptr[k] + (int)row.size();
    A.col_idx.insert(A.col_idx.end(), row.begin(), row.end());
  }
  A.val.assign(A.col_idx.size(), 0.0);
}

// pos_of, mod_uns_simple.f90:909-923 (-1 when absent)
inline int pos_of(const CSR& A, int i, int j) { return csr_find(A, i, j); }

// init_fields face weights, mod_uns_fields.f90:147-157
void init_lf(Case& cs) {
  const Mesh& m = cs.m;
  cs.lf.assign(m.nfaces, 1.0);
  for (int i = 0; i < m.nfaces; ++i) {
    int c1 = m.c1[i];
    if (c1 < 0) continue;
    int c0 = m.c0[i];
    double a[3], b[3];
    for (int k = 0; k < 3; ++k) {
      a[k] = cs.g.xf[3 * i + k] - cs.g.xc[3 * c0 + k];
      b[k] = cs.g.xc[3 * c1 + k] - cs.g.xf[3 * i + k];
    }
    double d0 = norm3(a), d1 = norm3(b);
    cs.lf[i] = d1 / (d0 + d1);
  }
}

// grad_scalar, mod_uns_fields.f90:355-374 (grad stride 3: grad(1:3,cell))
void grad_scalar(const Case& cs, const double* phif, double* grad, int gstride, int goff) {
  const Mesh& m = cs.m;
  for (int c = 0; c < m.ncells; ++c)
    for (int d = 0; d < 3; ++d) grad[gstride * c + goff + d] = 0.0;
  for (int i = 0; i < m.nfaces; ++i) {
    int c0 = m.c0[i];
    for (int d = 0; d < 3; ++d)
      grad[gstride * c0 + goff + d] = grad[gstride * c0 + goff + d] + phif[i] * cs.g.sf[3 * i + d];
    int c1 = m.c1[i];
    if (c1 >= 0)
      for (int d = 0; d < 3; ++d)
        grad[gstride * c1 + goff + d] = grad[gstride * c1 + goff + d] - phif[i] * cs.g.sf[3 * i + d];
  }
  for (int c = 0; c < m.ncells; ++c)
    for (int d = 0; d < 3; ++d) grad[gstride * c + goff + d] = grad[gstride * c + goff + d] / cs.g.vol[c];
}

// compute_gradients, mod_uns_fields.f90:164-258. gu is stored gu(comp,dir,cell)
// like the Fortran array. The temperature gradient gt (:219-237) is formed when
// the energy equation is solved (otherwise T is uniform and unused).
void compute_gradients(Case& cs) {
  const Mesh& m = cs.m;
  vector<double>& phif = cs.phif;
  phif.assign(m.nfaces, 0.0);
  for (int i = 0; i < m.nfaces; ++i) {
    int c0 = m.c0[i], c1 = m.c1[i];
    if (c1 >= 0)
      phif[i] = cs.lf[i] * cs.p[c0] + (1.0 - cs.lf[i]) * cs.p[c1];
    else
      phif[i] = bc_face_p(cs.bcs, i, cs.p[c0]);
  }
  grad_scalar(cs, phif.data(), cs.gp.data(), 3, 0);
  vector<double> tmp(3 * m.ncells);
  for (int comp = 0; comp < 3; ++comp) {
    for (int i = 0; i < m.nfaces; ++i) {
      int c0 = m.c0[i], c1 = m.c1[i];
      if (c1 >= 0)
        phif[i] = cs.lf[i] * cs.u[3 * c0 + comp] + (1.0 - cs.lf[i]) * cs.u[3 * c1 + comp];
      else {
        double uf[3];
        bc_face_vel(cs.bcs, i, &cs.g.xf[3 * i], &cs.g.sf[3 * i], &cs.u[3 * c0], uf);
        phif[i] = uf[comp];
      }
    }
    grad_scalar(cs, phif.data(), tmp.data(), 3, 0);
    for (int c = 0; c < m.ncells; ++c)
      for (int d = 0; d < 3; ++d) cs.gu[9 * c + comp + 3 * d] = tmp[3 * c + d];
  }
  if (cs.ctrl.energy) {
    for (int i = 0; i < m.nfaces; ++i) {
      int c0 = m.c0[i], c1 = m.c1[i];
      if (c1 >= 0) {
        phif[i] = cs.lf[i] * cs.T[c0] + (1.0 - cs.lf[i]) * cs.T[c1];
      } else {
        double tf, qf;
        bool neum;
        bc_face_T(cs.bcs, i, &cs.g.xf[3 * i], cs.T[c0], tf, qf, neum);
        phif[i] = tf;
      }
    }
    grad_scalar(cs, phif.data(), cs.gt.data(), 3, 0);
  }
}

// velocity_limiter, mod_uns_simple.f90:1346-1408
void velocity_limiter(Case& cs, int comp, vector<double>& psi) {
  const Mesh& m = cs.m;
  int N = m.ncells;
  vector<double> pmin(N), pmax(N);
  for (int i = 0; i < N; ++i) pmin[i] = pmax[i] = cs.u[3 * i + comp];
  for (int i = 0; i < m.nfaces; ++i) {
    int c0 = m.c0[i], c1 = m.c1[i];
    if (c1 >= 0) {
      pmin[c0] = std::min(pmin[c0], cs.u[3 * c1 + comp]);
      pmax[c0] = std::max(pmax[c0], cs.u[3 * c1 + comp]);
      pmin[c1] = std::min(pmin[c1], cs.u[3 * c0 + comp]);
      pmax[c1] = std::max(pmax[c1], cs.u[3 * c0 + comp]);
    } else if (cs.bcs.fgrp[i] >= 0) {
      double uf[3];
      bc_face_vel(cs.bcs, i, &cs.g.xf[3 * i], &cs.g.sf[3 * i], &cs.u[3 * c0], uf);
      pmin[c0] = std::min(pmin[c0], uf[comp]);
      pmax[c0] = std::max(pmax[c0], uf[comp]);
    }
  }
  psi.assign(N, 1.0);
  auto side = [&](int c, int i) {
    double uc = cs.u[3 * c + comp], d[3];
    for (int k = 0; k < 3; ++k) d[k] = cs.g.xf[3 * i + k] - cs.g.xc[3 * c + k];
    double gcomp[3] = {cs.gu[9 * c + comp], cs.gu[9 * c + comp + 3], cs.gu[9 * c + comp + 6]};
    double fr = uc + dot3(gcomp, d);
    double df = fr - uc;
    if (df > 0.0)
      psi[c] = std::min(psi[c], (pmax[c] - uc) / df);
    else if (df < 0.0)
      psi[c] = std::min(psi[c], (pmin[c] - uc) / df);
  };
  for (int i = 0; i < m.nfaces; ++i) {
    side(m.c0[i], i);
    if (m.c1[i] >= 0) side(m.c1[i], i);
  }
  for (int i = 0; i < N; ++i) psi[i] = std::max(0.0, std::min(1.0, psi[i]));
}

// momentum_assembly, mod_uns_simple.f90:928-1338, for a pure-fluid mesh
// (porosity 1, no porous/solid zones, no Boussinesq): the Beavers-Joseph,
// kink-pressure, Darcy-Forchheimer and solid-cell branches are inactive there.
void momentum_assembly(Case& cs, int comp) {
  const Mesh& m = cs.m;
  const MgpuCtrl& ctrl = cs.ctrl;
  CSR& A = cs.amat;
  int N = m.ncells;
  std::fill(A.val.begin(), A.val.end(), 0.0);
  cs.rhs.assign(N, 0.0);
  cs.ap.assign(N, 0.0);
  vector<double>& rhs = cs.rhs;
  vector<double>& ap = cs.ap;
  double sd = 0.0;
  if (ctrl.conv_blend > 0.0) velocity_limiter(cs, comp, cs.psi);
  const double POROSITY_FLOOR = 1.0e-8;
  for (int i = 0; i < m.nfaces; ++i) {
    int c1 = m.c1[i];
    if (c1 < 0) continue;
    int c0 = m.c0[i];
    double F = cs.flux[i];
    double dvec[3];
    for (int k = 0; k < 3; ++k) dvec[k] = cs.g.xc[3 * c1 + k] - cs.g.xc[3 * c0 + k];
    double dn = norm3(dvec);
    double mu_eff0 = ctrl.mu / std::max(1.0, POROSITY_FLOOR);
    double mu_eff1 = ctrl.mu / std::max(1.0, POROSITY_FLOOR);
    double mu_f = cs.lf[i] * mu_eff0 + (1.0 - cs.lf[i]) * mu_eff1;
    double D;
    double area = cs.g.area[i];
    if (ctrl.nonorth_corr > 0.0) {
      sd = dot3(&cs.g.sf[3 * i], dvec);
      D = mu_f * (area * area) / sd;
    } else {
      D = mu_f * area / dn;
    }
    double D_face = D;
    ap[c0] = ap[c0] + std::max(F, 0.0) + D_face;
    ap[c1] = ap[c1] + std::max(-F, 0.0) + D_face;
    int kd = pos_of(A, c0, c1);
    A.val[kd] = A.val[kd] - (D_face + std::max(-F, 0.0));
    kd = pos_of(A, c1, c0);
    A.val[kd] = A.val[kd] - (D_face + std::max(F, 0.0));
    if (ctrl.conv_blend > 0.0) {
      double dc;
      int cu = (F > 0.0) ? c0 : c1;
      double d[3];
      for (int k = 0; k < 3; ++k) d[k] = cs.g.xf[3 * i + k] - cs.g.xc[3 * cu + k];
      double gcomp[3] = {cs.gu[9 * cu + comp], cs.gu[9 * cu + comp + 3], cs.gu[9 * cu + comp + 6]};
      dc = cs.psi[cu] * dot3(gcomp, d);
      dc = ctrl.conv_blend * F * dc;
      rhs[c0] = rhs[c0] - dc;
      rhs[c1] = rhs[c1] + dc;
    }
    if (ctrl.nonorth_corr > 0.0) {
      double gf[3], t[3];
      for (int k = 0; k < 3; ++k) {
        gf[k] = cs.lf[i] * cs.gu[9 * c0 + comp + 3 * k] + (1.0 - cs.lf[i]) * cs.gu[9 * c1 + comp + 3 * k];
        t[k] = cs.g.sf[3 * i + k] - dvec[k] * ((area * area) / sd);
      }
      double noc = ctrl.nonorth_corr * mu_f * dot3(gf, t);
      rhs[c0] = rhs[c0] + noc;
      rhs[c1] = rhs[c1] - noc;
    }
    double pf = cs.lf[i] * cs.p[c0] + (1.0 - cs.lf[i]) * cs.p[c1];
    double Scomp = cs.g.sf[3 * i + comp];
    rhs[c0] = rhs[c0] - pf * Scomp;
    rhs[c1] = rhs[c1] + pf * Scomp;
  }
  for (int i = 0; i < m.nfaces; ++i) {
    int gi = cs.bcs.fgrp[i];
    if (gi < 0) continue;
    int c0 = m.c0[i];
    double uf[3];
    bc_face_vel(cs.bcs, i, &cs.g.xf[3 * i], &cs.g.sf[3 * i], &cs.u[3 * c0], uf);
    double pf = bc_face_p(cs.bcs, i, cs.p[c0]);
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = cs.g.xf[3 * i + k] - cs.g.xc[3 * c0 + k];
    double dw = norm3(d);
    double D = (ctrl.mu / std::max(1.0, POROSITY_FLOOR)) * cs.g.area[i] / dw;
    double F = ctrl.rho * dot3(uf, &cs.g.sf[3 * i]);
    switch (cs.bcs.gb[gi].btype) {
      case MGPU_BC_WALL:
      case MGPU_BC_SYMMETRY:
      case MGPU_BC_VINLET:
      case MGPU_BC_VINLET_PARAB:
      case MGPU_BC_SLIPWALL:
      case MGPU_BC_MASSINLET:
        ap[c0] = ap[c0] + D + std::max(F, 0.0);
        rhs[c0] = rhs[c0] + D * uf[comp] - F * uf[comp];
        break;
      case MGPU_BC_POUTLET:
      case MGPU_BC_OUTFLOW:
        ap[c0] = ap[c0] + std::max(F, 0.0);
        rhs[c0] = rhs[c0] - std::min(F, 0.0) * cs.u[3 * c0 + comp];
        break;
      case MGPU_BC_FARFIELD:
        if (F < 0.0) {
          ap[c0] = ap[c0] + D + std::max(F, 0.0);
          rhs[c0] = rhs[c0] + D * uf[comp] - F * uf[comp];
        } else {
          ap[c0] = ap[c0] + F;
        }
        break;
      case MGPU_BC_INTERFACE:  // mod_uns_simple.f90:1144-1176 (no slip / zhang variants)
        if (!cs.bcs.iface_p_dir) {
          ap[c0] = ap[c0] + D + std::max(F, 0.0);
          rhs[c0] = rhs[c0] + D * uf[comp] - F * uf[comp];
        } else {
          ap[c0] = ap[c0] + std::max(F, 0.0);
          rhs[c0] = rhs[c0] - std::min(F, 0.0) * cs.u[3 * c0 + comp];
        }
        break;
      default:
        break;
    }
    rhs[c0] = rhs[c0] - pf * cs.g.sf[3 * i + comp];
  }
  // Boussinesq buoyancy, mod_uns_simple.f90:1229-1240
  if (ctrl.boussinesq)
    for (int kk = 0; kk < N; ++kk)
      rhs[kk] = rhs[kk] - ctrl.rho * ctrl.beta * (cs.T[kk] - ctrl.tref) * ctrl.gravity[comp] * cs.g.vol[kk];
  if (ctrl.body_force[0] != 0.0 || ctrl.body_force[1] != 0.0 || ctrl.body_force[2] != 0.0)
    for (int kk = 0; kk < N; ++kk) rhs[kk] = rhs[kk] + ctrl.body_force[comp] * cs.g.vol[kk];
  if (cs.ts_order == 1) {
    for (int kk = 0; kk < N; ++kk) {
      double at = ctrl.rho * cs.g.vol[kk] / ctrl.dt;
      ap[kk] = ap[kk] + at;
      rhs[kk] = rhs[kk] + at * cs.u_old[3 * kk + comp];
    }
  } else if (cs.ts_order == 2) {
    for (int kk = 0; kk < N; ++kk) {
      double at = ctrl.rho * cs.g.vol[kk] / (2.0 * ctrl.dt);
      ap[kk] = ap[kk] + 3.0 * at;
      rhs[kk] = rhs[kk] + at * (4.0 * cs.u_old[3 * kk + comp] - cs.u_old_old[3 * kk + comp]);
    }
  }
  if (cs.ts_order > 0 && !cs.pimple) {  // PISO: no relaxation (ctrl%pimple = .false.)
    for (int kk = 0; kk < N; ++kk) A.val[pos_of(A, kk, kk)] = ap[kk];
  } else {
    for (int kk = 0; kk < N; ++kk) {
      A.val[pos_of(A, kk, kk)] = ap[kk] / ctrl.alpha_u;
      rhs[kk] = rhs[kk] + (1.0 - ctrl.alpha_u) / ctrl.alpha_u * ap[kk] * cs.u[3 * kk + comp];
    }
  }
}

// temperature_limiter, mod_uns_simple.f90:2302-2361 (Barth-Jespersen psi_T)
void temperature_limiter(const Case& cs, vector<double>& psi) {
  const Mesh& m = cs.m;
  const int N = m.ncells;
  vector<double> pmin(cs.T.begin(), cs.T.end()), pmax(cs.T.begin(), cs.T.end());
  for (int i = 0; i < m.nfaces; ++i) {
    int c0 = m.c0[i], c1 = m.c1[i];
    if (c1 >= 0) {
      pmin[c0] = std::min(pmin[c0], cs.T[c1]);
      pmax[c0] = std::max(pmax[c0], cs.T[c1]);
      pmin[c1] = std::min(pmin[c1], cs.T[c0]);
      pmax[c1] = std::max(pmax[c1], cs.T[c0]);
    } else if (cs.bcs.fgrp[i] >= 0) {
      double tf, qf;
      bool neum;
      bc_face_T(cs.bcs, i, &cs.g.xf[3 * i], cs.T[c0], tf, qf, neum);
      pmin[c0] = std::min(pmin[c0], tf);
      pmax[c0] = std::max(pmax[c0], tf);
    }
  }
  psi.assign(N, 1.0);
  auto side = [&](int c, int i) {
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = cs.g.xf[3 * i + k] - cs.g.xc[3 * c + k];
    const double tc = cs.T[c];
    const double fr = tc + dot3(&cs.gt[3 * c], d);
    const double df = fr - tc;
    if (df > 0.0)
      psi[c] = std::min(psi[c], (pmax[c] - tc) / df);
    else if (df < 0.0)
      psi[c] = std::min(psi[c], (pmin[c] - tc) / df);
  };
  for (int i = 0; i < m.nfaces; ++i) {
    side(m.c0[i], i);
    if (m.c1[i] >= 0) side(m.c1[i], i);
  }
  for (int i = 0; i < N; ++i) psi[i] = std::max(0.0, std::min(1.0, psi[i]));
}

// temperature_assembly, mod_uns_simple.f90:1748-2037, the branch this path
// takes: a clear fluid (porosity 1, no solid or porous zones, LTE, no
// dispersion), so k_eff = 1 k + 0 k_s and the dispersion terms add 0. Writes
// the CSR values into amat, rhs and ap (the unrelaxed ap_T).
void temperature_assembly(Case& cs) {
  const Mesh& m = cs.m;
  const MgpuCtrl& ctrl = cs.ctrl;
  const int N = m.ncells;
  CSR& A = cs.amat;
  std::fill(A.val.begin(), A.val.end(), 0.0);
  cs.rhs.assign(N, 0.0);
  cs.ap.assign(N, 0.0);
  vector<double>& rhs = cs.rhs;
  vector<double>& ap = cs.ap;
  vector<double> psiT;
  if (ctrl.conv_blend > 0.0) temperature_limiter(cs, psiT);
  // porosity = 1, k_s = 0: k_eff = 1 * k + (1 - 1) * 0
  const double k_eff = 1.0 * ctrl.k_cond + (1.0 - 1.0) * 0.0;
  double sd = 0.0;
  for (int i = 0; i < m.nfaces; ++i) {
    int c1 = m.c1[i], c0 = m.c0[i];
    if (c1 < 0) continue;
    const double FT = ctrl.cp * cs.flux[i];
    double dvec[3];
    for (int k = 0; k < 3; ++k) dvec[k] = cs.g.xc[3 * c1 + k] - cs.g.xc[3 * c0 + k];
    const double dn = norm2_scaled(dvec, 3);
    double kf = cs.lf[i] * k_eff + (1.0 - cs.lf[i]) * k_eff;
    kf = kf + (cs.lf[i] * 0.0 + (1.0 - cs.lf[i]) * 0.0);  // dispersion of a clear fluid
    const double area = cs.g.area[i];
    double DT;
    if (ctrl.nonorth_corr > 0.0) {
      sd = dot3(&cs.g.sf[3 * i], dvec);
      DT = kf * (area * area) / sd;
    } else {
      DT = kf * area / dn;
    }
    ap[c0] = ap[c0] + std::max(FT, 0.0) + DT;
    ap[c1] = ap[c1] + std::max(-FT, 0.0) + DT;
    int kd = pos_of(A, c0, c1);
    A.val[kd] = A.val[kd] - (DT + std::max(-FT, 0.0));
    kd = pos_of(A, c1, c0);
    A.val[kd] = A.val[kd] - (DT + std::max(FT, 0.0));
    if (ctrl.conv_blend > 0.0) {
      double dc;
      if (FT > 0.0) {
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = cs.g.xf[3 * i + k] - cs.g.xc[3 * c0 + k];
        dc = psiT[c0] * dot3(&cs.gt[3 * c0], d);
      } else {
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = cs.g.xf[3 * i + k] - cs.g.xc[3 * c1 + k];
        dc = psiT[c1] * dot3(&cs.gt[3 * c1], d);
      }
      dc = ctrl.conv_blend * FT * dc;
      rhs[c0] = rhs[c0] - dc;
      rhs[c1] = rhs[c1] + dc;
    }
    if (ctrl.nonorth_corr > 0.0) {
      double gf[3], w[3];
      const double a2 = area * area / sd;
      for (int k = 0; k < 3; ++k) {
        gf[k] = cs.lf[i] * cs.gt[3 * c0 + k] + (1.0 - cs.lf[i]) * cs.gt[3 * c1 + k];
        w[k] = cs.g.sf[3 * i + k] - dvec[k] * a2;
      }
      const double noc = ctrl.nonorth_corr * kf * dot3(gf, w);
      rhs[c0] = rhs[c0] + noc;
      rhs[c1] = rhs[c1] - noc;
    }
  }
  for (int i = 0; i < m.nfaces; ++i) {
    if (cs.bcs.fgrp[i] < 0) continue;
    const int c0 = m.c0[i];
    double T_face, q_face;
    bool is_neumann;
    bc_face_T(cs.bcs, i, &cs.g.xf[3 * i], cs.T[c0], T_face, q_face, is_neumann);
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = cs.g.xf[3 * i + k] - cs.g.xc[3 * c0 + k];
    const double dw = norm2_scaled(d, 3);
    double kf = 1.0 * ctrl.k_cond + (1.0 - 1.0) * 0.0;
    kf = kf + 0.0;  // dispersion of a clear fluid
    const double DT = kf * cs.g.area[i] / dw;
    const double FT = ctrl.cp * cs.flux[i];
    if (!is_neumann) {
      ap[c0] = ap[c0] + DT + std::max(FT, 0.0);
      rhs[c0] = rhs[c0] + DT * T_face - std::min(FT, 0.0) * T_face;
    } else {
      if (std::fabs(q_face) > 0.0) rhs[c0] = rhs[c0] + q_face * cs.g.area[i];
      const int bt = cs.bcs.gb[cs.bcs.fgrp[i]].btype;
      if (bt == MGPU_BC_POUTLET || bt == MGPU_BC_OUTFLOW) ap[c0] = ap[c0] + std::max(FT, 0.0);
    }
  }
  // time term: (rho cp)_eff = 1 rho cp + (1 - 1) rho_s cp_s
  if (cs.ts_order == 1) {
    for (int kk = 0; kk < N; ++kk) {
      const double at = (1.0 * ctrl.rho * ctrl.cp + (1.0 - 1.0) * 0.0 * 0.0) * cs.g.vol[kk] / ctrl.dt;
      ap[kk] = ap[kk] + at;
      rhs[kk] = rhs[kk] + at * cs.T_old[kk];
    }
  } else if (cs.ts_order == 2) {
    for (int kk = 0; kk < N; ++kk) {
      const double at = (1.0 * ctrl.rho * ctrl.cp + (1.0 - 1.0) * 0.0 * 0.0) * cs.g.vol[kk] / (2.0 * ctrl.dt);
      ap[kk] = ap[kk] + 3.0 * at;
      rhs[kk] = rhs[kk] + at * (4.0 * cs.T_old[kk] - cs.T_old_old[kk]);
    }
  }
  if (cs.ts_order > 0 && !cs.pimple) {
    for (int kk = 0; kk < N; ++kk) A.val[pos_of(A, kk, kk)] = ap[kk];
  } else {
    for (int kk = 0; kk < N; ++kk) {
      A.val[pos_of(A, kk, kk)] = ap[kk] / ctrl.alpha_u;
      rhs[kk] = rhs[kk] + (1.0 - ctrl.alpha_u) / ctrl.alpha_u * ap[kk] * cs.T[kk];
    }
  }
}

// flux_rhiechow, mod_uns_simple.f90:1413-1450
void flux_rhiechow(Case& cs) {
  const Mesh& m = cs.m;
  for (int i = 0; i < m.nfaces; ++i) {
    int c1 = m.c1[i], c0 = m.c0[i];
    const double* sf = &cs.g.sf[3 * i];
    if (c1 < 0) {
      double uf[3];
      bc_face_vel(cs.bcs, i, &cs.g.xf[3 * i], sf, &cs.u[3 * c0], uf);
      cs.flux[i] = cs.ctrl.rho * dot3(uf, sf);
      continue;
    }
    double lf = cs.lf[i], ufl[3], gpl[3], dvec[3];
    for (int k = 0; k < 3; ++k) {
      ufl[k] = lf * cs.u[3 * c0 + k] + (1.0 - lf) * cs.u[3 * c1 + k];
      gpl[k] = lf * cs.gp[3 * c0 + k] + (1.0 - lf) * cs.gp[3 * c1 + k];
      dvec[k] = cs.g.xc[3 * c1 + k] - cs.g.xc[3 * c0 + k];
    }
    double dn = norm3(dvec);
    double pfgrad_n = (cs.p[c1] - cs.p[c0]) / dn;
    double dbf = lf * cs.g.vol[c0] / cs.apc[c0] + (1.0 - lf) * cs.g.vol[c1] / cs.apc[c1];
    cs.flux[i] = cs.ctrl.rho * (dot3(ufl, sf) + dbf * (dot3(gpl, sf) - pfgrad_n * dot3(dvec, sf) / dn));
  }
}

// outflow_mass_sums / outflow_mass_scale, mod_uns_simple.f90:1463-1531
void outflow_mass_rescale(Case& cs) {
  const Mesh& m = cs.m;
  double m_req = 0.0, m_out = 0.0, area_out = 0.0;
  for (int i = 0; i < m.nfaces; ++i) {
    if (m.c1[i] >= 0) continue;
    int gi = cs.bcs.fgrp[i];
    if (gi < 0) continue;
    int bt = cs.bcs.gb[gi].btype;
    if (bt == MGPU_BC_OUTFLOW) {
      m_out = m_out + cs.flux[i];
      area_out = area_out + cs.g.area[i];
    } else if (bt != MGPU_BC_POUTLET && bt != MGPU_BC_FARFIELD) {
      m_req = m_req - cs.flux[i];
    }
  }
  if (area_out <= 0.0 || m_req <= 0.0) return;
  bool scaled = m_out > 1.0e-2 * m_req;
  double beta = scaled ? m_req / m_out : 0.0;
  for (int i = 0; i < m.nfaces; ++i) {
    if (m.c1[i] >= 0) continue;
    int gi = cs.bcs.fgrp[i];
    if (gi < 0 || cs.bcs.gb[gi].btype != MGPU_BC_OUTFLOW) continue;
    cs.flux[i] = scaled ? beta * cs.flux[i] : m_req * cs.g.area[i] / area_out;
  }
}

// ppe_assembly, mod_uns_simple.f90:1552-1644 (the one-rank ppe_assembly_mpi,
// mod_uns_simple_mpi.f90:882-968, is identical for the boundary types here)
void ppe_assembly(Case& cs) {
  const Mesh& m = cs.m;
  CSR& A = cs.pmat;
  std::fill(A.val.begin(), A.val.end(), 0.0);
  cs.rhs.assign(m.ncells, 0.0);
  vector<double>& rhs = cs.rhs;
  double rho = cs.ctrl.rho;
  // the transient drivers assemble with ppe_assembly_mpi at one rank
  const bool mpi = cs.ts_order > 0;
  auto dirichlet = [&](int i) { return mpi ? ppe_dirichlet_mpi(cs.bcs, i) : bc_face_p_dirichlet(cs.bcs, i); };
  for (int i = 0; i < m.nfaces; ++i) {
    int c1 = m.c1[i], c0 = m.c0[i];
    if (c1 < 0) {
      if (cs.bcs.fgrp[i] >= 0 && dirichlet(i)) {
        double dbf = cs.g.vol[c0] / cs.apc[c0];
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = cs.g.xf[3 * i + k] - cs.g.xc[3 * c0 + k];
        double dn = norm3(d);
        double af = rho * dbf * cs.g.area[i] / dn;
        int kd = pos_of(A, c0, c0);
        A.val[kd] = A.val[kd] + af;
      }
      rhs[c0] = rhs[c0] - cs.flux[i];
      continue;
    }
    double lf = cs.lf[i];
    double dbf = lf * cs.g.vol[c0] / cs.apc[c0] + (1.0 - lf) * cs.g.vol[c1] / cs.apc[c1];
    double dv[3];
    for (int k = 0; k < 3; ++k) dv[k] = cs.g.xc[3 * c1 + k] - cs.g.xc[3 * c0 + k];
    double dn = norm3(dv);
    double af = rho * dbf * cs.g.area[i] / dn;
    int kd = pos_of(A, c0, c0);
    A.val[kd] = A.val[kd] + af;
    kd = pos_of(A, c0, c1);
    A.val[kd] = A.val[kd] - af;
    kd = pos_of(A, c1, c1);
    A.val[kd] = A.val[kd] + af;
    kd = pos_of(A, c1, c0);
    A.val[kd] = A.val[kd] - af;
    rhs[c0] = rhs[c0] - cs.flux[i];
    rhs[c1] = rhs[c1] + cs.flux[i];
  }
  bool has_pdir = false;
  for (int i = 0; i < m.nfaces; ++i)
    if (m.c1[i] < 0 && cs.bcs.fgrp[i] >= 0 && dirichlet(i)) has_pdir = true;
  if (!has_pdir) {
    for (int k = A.row_ptr[0]; k < A.row_ptr[1]; ++k) A.val[k] = (A.col_idx[k] == 0) ? 1.0 : 0.0;
    for (int kk = 1; kk < A.nrows; ++kk) {
      int kd = pos_of(A, kk, 0);
      if (kd >= 0) A.val[kd] = 0.0;
    }
    rhs[0] = 0.0;
  }
}

// correct_fields, mod_uns_simple.f90:1649-1739
void correct_fields(Case& cs) {
  const Mesh& m = cs.m;
  const double* pp = cs.pp.data();
  cs.phif.assign(m.nfaces, 0.0);
  for (int i = 0; i < m.nfaces; ++i) {
    int c1 = m.c1[i];
    if (c1 >= 0) {
      cs.phif[i] = cs.lf[i] * pp[m.c0[i]] + (1.0 - cs.lf[i]) * pp[c1];
    } else {
      if (cs.bcs.fgrp[i] >= 0 && bc_face_p_dirichlet(cs.bcs, i)) {
        cs.phif[i] = 0.0;
        continue;
      }
      cs.phif[i] = pp[m.c0[i]];
    }
  }
  cs.dpp.assign(3 * m.ncells, 0.0);
  grad_scalar(cs, cs.phif.data(), cs.dpp.data(), 3, 0);
  for (int i = 0; i < m.ncells; ++i)
    for (int k = 0; k < 3; ++k) cs.u[3 * i + k] = cs.u[3 * i + k] - (cs.g.vol[i] / cs.apc[i]) * cs.dpp[3 * i + k];
  if (cs.ts_order > 0)
    for (int i = 0; i < m.ncells; ++i) cs.p[i] = cs.p[i] + pp[i];
  else
    for (int i = 0; i < m.ncells; ++i) cs.p[i] = cs.p[i] + cs.ctrl.alpha_p * pp[i];
  double rho = cs.ctrl.rho;
  // every driver (the transient ones included) corrects the fluxes with the
  // serial correct_fields and its bc_face_p_dirichlet rule, mod_uns_simple.f90:1703-1724
  // (mod_uns_simple_mpi.f90:187, 457, 740)
  for (int i = 0; i < m.nfaces; ++i) {
    int c1 = m.c1[i], c0 = m.c0[i];
    if (c1 < 0) {
      if (cs.bcs.fgrp[i] >= 0 && bc_face_p_dirichlet(cs.bcs, i)) {
        double dbf = cs.g.vol[c0] / cs.apc[c0];
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = cs.g.xf[3 * i + k] - cs.g.xc[3 * c0 + k];
        double dn = norm3(d);
        double af = rho * dbf * cs.g.area[i] / dn;
        cs.flux[i] = cs.flux[i] + af * pp[c0];
      }
      continue;
    }
    double lf = cs.lf[i];
    double dbf = lf * cs.g.vol[c0] / cs.apc[c0] + (1.0 - lf) * cs.g.vol[c1] / cs.apc[c1];
    double dv[3];
    for (int k = 0; k < 3; ++k) dv[k] = cs.g.xc[3 * c1 + k] - cs.g.xc[3 * c0 + k];
    double dn = norm3(dv);
    double af = rho * dbf * cs.g.area[i] / dn;
    cs.flux[i] = cs.flux[i] - af * (pp[c1] - pp[c0]);
  }
}

// nan_scan, mod_uns_simple.f90:2375-2426 (fields u_x u_y u_z p T T_s; T and
// T_s are identically zero on this path and are always finite)
int nan_scan(const Case& cs, int& field, int& cell, double& val, int& kind) {
  field = 0;
  cell = 0;
  val = 0.0;
  kind = 0;
  for (int ic = 0; ic < cs.m.ncells; ++ic) {
    double v5[5] = {cs.u[3 * ic], cs.u[3 * ic + 1], cs.u[3 * ic + 2], cs.p[ic], cs.T[ic]};
    for (int f = 0; f < 5; ++f)
      if (!std::isfinite(v5[f])) {
        field = f + 1;
        cell = ic + 1;
        val = v5[f];
        kind = std::isnan(v5[f]) ? 1 : 2;
        return 1;
      }
  }
  return 0;
}

double flux_reference(const Case& cs) {
  double uscale = 0.0, area_btot = 0.0;
  for (const Group& gb : cs.bcs.gb) {
    uscale = std::max(std::max(std::max(uscale, norm3(gb.lid_vel)), norm3(gb.uvel)), gb.uspeed);
    for (int f : gb.faces) area_btot = area_btot + cs.g.area[f];
  }
  if (uscale <= 0.0) uscale = 1.0;
  if (area_btot <= 0.0) area_btot = 1.0;
  return cs.ctrl.rho * uscale * area_btot;
}

double max_imbalance(const Case& cs) {
  const Mesh& m = cs.m;
  vector<double> imbalc(m.ncells, 0.0);
  for (int i = 0; i < m.nfaces; ++i) {
    imbalc[m.c0[i]] = imbalc[m.c0[i]] + cs.flux[i];
    if (m.c1[i] >= 0) imbalc[m.c1[i]] = imbalc[m.c1[i]] - cs.flux[i];
  }
  double mx = 0.0;
  for (double v : imbalc) mx = std::max(mx, std::fabs(v));
  return mx;
}

void solve_momentum(Case& cs, int comp, int norm_mode, int& itl, double& resl, int& ierr) {
  int N = cs.m.ncells;
  vector<double> x(N);
  for (int i = 0; i < N; ++i) x[i] = cs.u[3 * i + comp];
  int pk = cs.ctrl.mom_solver == MGPU_MOM_JACOBI ? 1 : 0;
  bicgstab(cs.amat, cs.rhs.data(), x.data(), cs.ctrl.lin_tol, cs.ctrl.lin_max, itl, resl, ierr, pk, Norm{norm_mode});
  for (int i = 0; i < N; ++i) cs.u[3 * i + comp] = x[i];
}

void solve_ppe(Case& cs, int norm_mode, int& itl, double& resl, int& ierr) {
  int N = cs.m.ncells;
  cs.pp.assign(N, 0.0);
  int pk = cs.ctrl.ppe_precond == MGPU_PPE_IC0 ? 2 : (cs.ctrl.ppe_precond == MGPU_PPE_ILU0 ? 0 : 1);
  pcg(cs.pmat, cs.rhs.data(), cs.pp.data(), cs.ctrl.lin_tol, cs.ctrl.lin_max, itl, resl, ierr, pk, Norm{norm_mode});
}

// The temperature solve: bicgstab_ilu0 on amat from the current T (the
// reference's, mod_uns_simple.f90:205 / mod_uns_simple_mpi.f90:469, 752); the
// preconditioner follows the momentum solver like the momentum solves.
void solve_temperature(Case& cs, int norm_mode, int& itl, double& resl, int& ierr) {
  int pk = cs.ctrl.mom_solver == MGPU_MOM_JACOBI ? 1 : 0;
  bicgstab(cs.amat, cs.rhs.data(), cs.T.data(), cs.ctrl.lin_tol, cs.ctrl.lin_max, itl, resl, ierr, pk, Norm{norm_mode});
}

// Energy step of the drivers: Tprev, assembly, solve into record slot ns;
// dT_max = max |T - Tprev|. Returns false on a breakdown.
bool energy_step(Case& cs, int norm_mode, MgpuIterRec& rec, int& ns, int& itl_max, double& dT_max) {
  const int N = cs.m.ncells;
  vector<double> Tprev = cs.T;
  temperature_assembly(cs);
  int itl, ierr;
  double resl;
  solve_temperature(cs, norm_mode, itl, resl, ierr);
  if (ns < MGPU_MAXSOLVE) {
    rec.lin_it[ns] = itl;
    rec.lin_res[ns] = resl;
    rec.lin_ierr[ns] = ierr;
    ++ns;
  }
  if (ierr == 2) return false;
  itl_max = std::max(itl_max, itl);
  dT_max = 0.0;
  for (int i = 0; i < N; ++i) dT_max = std::max(dT_max, std::fabs(cs.T[i] - Tprev[i]));
  return true;
}

// simple_run, mod_uns_simple.f90:88-288
int simple_run(Case& cs, int nsteps, MgpuIterRec* log, int logcap, int* nrec) {
  const MgpuCtrl& ctrl = cs.ctrl;
  int N = cs.m.ncells;
  double flux_ref = flux_reference(cs);
  std::fill(cs.apc.begin(), cs.apc.end(), 1.0);
  cs.ts_order = 0;
  compute_gradients(cs);
  int it_max = ctrl.outer_max;
  if (nsteps > 0) it_max = std::min(it_max, nsteps);
  *nrec = 0;
  for (int it = 1; it <= it_max; ++it) {
    vector<double> uo = cs.u;
    MgpuIterRec rec;
    std::memset(&rec, 0, sizeof(rec));
    rec.it = it;
    int itl_max = 0, itl, ierr;
    double ressum = 0.0, resl;
    if (ctrl.inlet_ramp > 1) {
      double f = (double)it / (double)ctrl.inlet_ramp;
      cs.bcs.inlet_ramp = std::max(0.0, std::min(1.0, f));
      cs.bcs.pval_ramp = std::max(0.0, std::min(1.0, f));
    }
    for (int comp = 0; comp < 3; ++comp) {
      momentum_assembly(cs, comp);
      solve_momentum(cs, comp, 0, itl, resl, ierr);
      rec.lin_it[comp] = itl;
      rec.lin_res[comp] = resl;
      rec.lin_ierr[comp] = ierr;
      if (ierr == 2) return 20;
      itl_max = std::max(itl_max, itl);
      ressum = ressum + resl;
    }
    for (int i = 0; i < N; ++i) cs.apc[i] = cs.ap[i] / ctrl.alpha_u;
    compute_gradients(cs);
    flux_rhiechow(cs);
    outflow_mass_rescale(cs);
    ppe_assembly(cs);
    solve_ppe(cs, 0, itl, resl, ierr);
    rec.lin_it[3] = itl;
    rec.lin_res[3] = resl;
    rec.lin_ierr[3] = ierr;
    rec.nsolve = 4;
    if (ierr == 2) return 21;
    itl_max = std::max(itl_max, itl);
    correct_fields(cs);
    // 5b. temperature equation (without ctrl.energy T is uniform with no
    // thermal boundary: the reference's solve then returns at once)
    double dT_max = 0.0;
    if (ctrl.energy) {
      int ns = 4;
      if (!energy_step(cs, 0, rec, ns, itl_max, dT_max)) return 22;
      rec.nsolve = ns;
    }
    int fld, cell, kind;
    double val;
    if (nan_scan(cs, fld, cell, val, kind)) return 60;
    double imbal = max_imbalance(cs) / flux_ref;
    double du_max = 0.0;
    for (int i = 0; i < 3 * N; ++i) du_max = std::max(du_max, std::fabs(cs.u[i] - uo[i]));
    rec.itl_max = itl_max;
    rec.imbal = imbal;
    rec.du_max = du_max;
    rec.dT_max = dT_max;
    rec.ressum = ressum;
    if (log && *nrec < logcap) log[*nrec] = rec;
    ++*nrec;
    if (imbal < ctrl.outer_tol && du_max < ctrl.outer_tol && dT_max < ctrl.outer_tol) break;
  }
  return 0;
}

// piso_run_mpi at one rank, mod_uns_simple_mpi.f90:298-571
int piso_run(Case& cs, int nsteps, MgpuIterRec* log, int logcap, int* nrec) {
  const MgpuCtrl& ctrl = cs.ctrl;
  int N = cs.m.ncells;
  *nrec = 0;
  if (!ctrl.transient) return 30;
  if (ctrl.dt <= 0.0) return 31;
  int n_steps = std::max(1, ctrl.n_time_max);
  if (nsteps > 0) n_steps = std::min(n_steps, nsteps);
  double flux_ref = flux_reference(cs);
  std::fill(cs.apc.begin(), cs.apc.end(), 1.0);
  compute_gradients(cs);
  flux_rhiechow(cs);
  double t_now = 0.0;
  for (int it = 1; it <= n_steps; ++it) {
    cs.u_old_old = cs.u_old;
    cs.u_old = cs.u;
    cs.T_old_old = cs.T_old;
    cs.T_old = cs.T;
    cs.ts_order = (it == 1 || ctrl.time_scheme == 1) ? 1 : 2;
    MgpuIterRec rec;
    std::memset(&rec, 0, sizeof(rec));
    rec.it = it;
    int itl_max = 0, itl, ierr;
    double ressum = 0.0, resl;
    for (int comp = 0; comp < 3; ++comp) {
      momentum_assembly(cs, comp);
      solve_momentum(cs, comp, 1, itl, resl, ierr);
      rec.lin_it[comp] = itl;
      rec.lin_res[comp] = resl;
      rec.lin_ierr[comp] = ierr;
      if (ierr == 2) return 33;
      itl_max = std::max(itl_max, itl);
      ressum = ressum + resl;
    }
    cs.apc = cs.ap;
    compute_gradients(cs);
    flux_rhiechow(cs);
    outflow_mass_rescale(cs);
    int ns = 3;
    for (int icorr = 1; icorr <= ctrl.n_correct; ++icorr) {
      ppe_assembly(cs);
      solve_ppe(cs, 1, itl, resl, ierr);
      if (ns < MGPU_MAXSOLVE) {
        rec.lin_it[ns] = itl;
        rec.lin_res[ns] = resl;
        rec.lin_ierr[ns] = ierr;
        ++ns;
      }
      if (ierr == 2) return 34;
      itl_max = std::max(itl_max, itl);
      correct_fields(cs);
    }
    // 4b. temperature equation (mod_uns_simple_mpi.f90:467-479)
    if (ctrl.energy && !energy_step(cs, 1, rec, ns, itl_max, rec.dT_max)) return 35;
    rec.nsolve = ns;
    t_now = t_now + ctrl.dt;
    double imbal = max_imbalance(cs) / flux_ref;
    double du_max = 0.0;
    for (int i = 0; i < 3 * N; ++i) du_max = std::max(du_max, std::fabs(cs.u[i] - cs.u_old[i]));
    du_max = du_max / ctrl.dt;
    double umax = 0.0;
    for (int i = 0; i < N; ++i) umax = std::max(umax, norm3(&cs.u[3 * i]));
    double cfl = 0.0;
    for (int i = 0; i < N; ++i) {
      double dt_dx = umax * ctrl.dt / std::pow(cs.g.vol[i], 1.0 / 3.0);
      if (dt_dx > cfl) cfl = dt_dx;
    }
    int fld, cell, kind;
    double val;
    if (nan_scan(cs, fld, cell, val, kind)) return 60;
    rec.itl_max = itl_max;
    rec.imbal = imbal;
    rec.du_max = du_max;
    rec.ressum = ressum;
    rec.umax = umax;
    rec.cfl_max = cfl;
    rec.t_now = t_now;
    if (log && *nrec < logcap) log[*nrec] = rec;
    ++*nrec;
  }
  return 0;
}

// pimple_run_mpi at one rank, mod_uns_simple_mpi.f90:580-850: one history
// shift per time step, n_outer_iter outer iterations of (relaxed momentum,
// apc = ap / alpha_u, gradients, Rhie-Chow, outflow rescale, n_correct PPE
// solves and corrections), then the step's diagnostics. The record keeps the
// last outer iteration's solves; itl_max and ressum run over all of them.
int pimple_run_body(Case& cs, int nsteps, MgpuIterRec* log, int logcap, int* nrec) {
  const MgpuCtrl& ctrl = cs.ctrl;
  int N = cs.m.ncells;
  *nrec = 0;
  if (!ctrl.transient) return 50;
  if (ctrl.dt <= 0.0) return 51;
  int n_steps = std::max(1, ctrl.n_time_max);
  if (nsteps > 0) n_steps = std::min(n_steps, nsteps);
  const int n_outer = std::max(1, ctrl.n_outer_iter);
  double flux_ref = flux_reference(cs);
  std::fill(cs.apc.begin(), cs.apc.end(), 1.0);
  compute_gradients(cs);
  flux_rhiechow(cs);
  double t_now = 0.0;
  for (int it = 1; it <= n_steps; ++it) {
    cs.u_old_old = cs.u_old;
    cs.u_old = cs.u;
    cs.T_old_old = cs.T_old;
    cs.T_old = cs.T;
    cs.ts_order = (it == 1 || ctrl.time_scheme == 1) ? 1 : 2;
    MgpuIterRec rec;
    std::memset(&rec, 0, sizeof(rec));
    rec.it = it;
    int itl_max = 0, itl, ierr;
    double ressum = 0.0, resl;
    int ns = 3;
    for (int iouter = 1; iouter <= n_outer; ++iouter) {
      for (int comp = 0; comp < 3; ++comp) {
        momentum_assembly(cs, comp);
        solve_momentum(cs, comp, 1, itl, resl, ierr);
        rec.lin_it[comp] = itl;
        rec.lin_res[comp] = resl;
        rec.lin_ierr[comp] = ierr;
        if (ierr == 2) return 53;
        itl_max = std::max(itl_max, itl);
        ressum = ressum + resl;
      }
      for (int i = 0; i < N; ++i) cs.apc[i] = cs.ap[i] / ctrl.alpha_u;
      compute_gradients(cs);
      flux_rhiechow(cs);
      outflow_mass_rescale(cs);
      ns = 3;
      for (int icorr = 1; icorr <= ctrl.n_correct; ++icorr) {
        ppe_assembly(cs);
        solve_ppe(cs, 1, itl, resl, ierr);
        if (ns < MGPU_MAXSOLVE) {
          rec.lin_it[ns] = itl;
          rec.lin_res[ns] = resl;
          rec.lin_ierr[ns] = ierr;
          ++ns;
        }
        if (ierr == 2) return 54;
        itl_max = std::max(itl_max, itl);
        correct_fields(cs);
      }
    }
    // temperature once per step, after the outer iterations (mod_uns_simple_mpi.f90:750-759)
    if (ctrl.energy && !energy_step(cs, 1, rec, ns, itl_max, rec.dT_max)) return 55;
    rec.nsolve = ns;
    t_now = t_now + ctrl.dt;
    double imbal = max_imbalance(cs) / flux_ref;
    double du_max = 0.0;
    for (int i = 0; i < 3 * N; ++i) du_max = std::max(du_max, std::fabs(cs.u[i] - cs.u_old[i]));
    du_max = du_max / ctrl.dt;
    double umax = 0.0;
    for (int i = 0; i < N; ++i) umax = std::max(umax, norm3(&cs.u[3 * i]));
    double cfl = 0.0;
    for (int i = 0; i < N; ++i) {
      double dt_dx = umax * ctrl.dt / std::pow(cs.g.vol[i], 1.0 / 3.0);
      if (dt_dx > cfl) cfl = dt_dx;
    }
    int fld, cell, kind;
    double val;
    if (nan_scan(cs, fld, cell, val, kind)) return 60;
    rec.itl_max = itl_max;
    rec.imbal = imbal;
    rec.du_max = du_max;
    rec.ressum = ressum;
    rec.umax = umax;
    rec.cfl_max = cfl;
    rec.t_now = t_now;
    if (log && *nrec < logcap) log[*nrec] = rec;
    ++*nrec;
  }
  return 0;
}

int pimple_run(Case& cs, int nsteps, MgpuIterRec* log, int logcap, int* nrec) {
  cs.pimple = true;
  const int ier = pimple_run_body(cs, nsteps, log, logcap, nrec);
  cs.pimple = false;
  return ier;
}

bool load_mesh(const MgpuMesh* in, Mesh& m) {
  if (!in || in->ncells <= 0 || in->nfaces <= 0 || in->nnodes <= 0) return false;
  m.nnodes = in->nnodes;
  m.nfaces = in->nfaces;
  m.ncells = in->ncells;
  m.x.assign(in->x, in->x + 3 * (long)m.nnodes);
  m.fptr.assign(in->fnode_ptr, in->fnode_ptr + m.nfaces + 1);
  m.fnodes.resize(m.fptr[m.nfaces]);
  for (int j = 0; j < m.fptr[m.nfaces]; ++j) {
    m.fnodes[j] = in->fnodes[j] - 1;
    if (m.fnodes[j] < 0 || m.fnodes[j] >= m.nnodes) return false;
  }
  m.c0.resize(m.nfaces);
  m.c1.resize(m.nfaces);
  m.zone.assign(in->zone, in->zone + m.nfaces);
  for (int i = 0; i < m.nfaces; ++i) {
    m.c0[i] = in->c0[i] - 1;
    m.c1[i] = in->c1[i] - 1;
    if (m.c0[i] < 0 || m.c0[i] >= m.ncells || m.c1[i] < -1 || m.c1[i] >= m.ncells) return false;
  }
  return true;
}

void to_csr(int n, const int32_t* rp, const int32_t* ci, const double* v, CSR& A) {
  A.nrows = n;
  A.row_ptr.resize(n + 1);
  for (int i = 0; i <= n; ++i) A.row_ptr[i] = rp[i] - 1;
  int nnz = A.row_ptr[n];
  A.col_idx.resize(nnz);
  for (int k = 0; k < nnz; ++k) A.col_idx[k] = ci[k] - 1;
  A.val.assign(v, v + nnz);
}

}  // namespace

extern "C" {

struct OrcCase {
  Case cs;
};

int orc_case_create(const MgpuMesh* mesh, const MgpuCtrl* ctrl, OrcCase** out, int* ier) {
  *out = nullptr;
  if (ier) *ier = 0;
  OrcCase* oc = new OrcCase();
  Case& cs = oc->cs;
  if (!load_mesh(mesh, cs.m)) {
    delete oc;
    return MGPU_E_MESH;
  }
  cs.ctrl = *ctrl;
  build_connectivity(cs.m, cs.conn);
  compute_geometry(cs.m, cs.g);
  int e = build_bc(cs.m, cs.ctrl, cs.bcs);
  if (e != 0) {
    if (ier) *ier = e;
    delete oc;
    return MGPU_E_BC;
  }
  int N = cs.m.ncells, F = cs.m.nfaces;
  cs.bcs.iface_vel.assign(3 * (size_t)F, 0.0);  // build_bc's zero-initialised interface data
  cs.bcs.iface_p.assign(F, 0.0);
  cs.bcs.iface_T.assign(F, 0.0);
  cs.bcs.iface_q.assign(F, 0.0);
  cs.bcs.iface_T_mode.assign(F, 0);
  cs.u.assign(3 * N, 0.0);
  cs.p.assign(N, 0.0);
  cs.gp.assign(3 * N, 0.0);
  cs.gu.assign(9 * N, 0.0);
  cs.flux.assign(F, 0.0);
  cs.apc.assign(N, 1.0);
  cs.u_old.assign(3 * N, 0.0);
  cs.u_old_old.assign(3 * N, 0.0);
  cs.T.assign(N, 0.0);
  cs.T_old.assign(N, 0.0);
  cs.T_old_old.assign(N, 0.0);
  cs.gt.assign(3 * N, 0.0);
  init_lf(cs);
  build_cell_csr(cs.m, cs.conn, cs.amat);
  cs.pmat = cs.amat;
  *out = oc;
  return 0;
}

int orc_case_destroy(OrcCase* c) {
  delete c;
  return 0;
}

int orc_fields_upload(OrcCase* c, const double* u, const double* p, const double* flux, const double* u_old,
                      const double* u_old_old) {
  Case& cs = c->cs;
  int N = cs.m.ncells;
  if (u) cs.u.assign(u, u + 3 * N);
  if (p) cs.p.assign(p, p + N);
  if (flux) cs.flux.assign(flux, flux + cs.m.nfaces);
  if (u_old) cs.u_old.assign(u_old, u_old + 3 * N);
  if (u_old_old) cs.u_old_old.assign(u_old_old, u_old_old + 3 * N);
  return 0;
}

int orc_fields_download(OrcCase* c, double* u, double* p, double* flux, double* gp, double* gu, double* apc) {
  Case& cs = c->cs;
  if (u) std::copy(cs.u.begin(), cs.u.end(), u);
  if (p) std::copy(cs.p.begin(), cs.p.end(), p);
  if (flux) std::copy(cs.flux.begin(), cs.flux.end(), flux);
  if (gp) std::copy(cs.gp.begin(), cs.gp.end(), gp);
  if (gu) std::copy(cs.gu.begin(), cs.gu.end(), gu);
  if (apc) std::copy(cs.apc.begin(), cs.apc.end(), apc);
  return 0;
}

int orc_temperature_upload(OrcCase* c, const double* T, const double* T_old, const double* T_old_old) {
  Case& cs = c->cs;
  const int N = cs.m.ncells;
  if (T) cs.T.assign(T, T + N);
  cs.T_old = T_old ? vector<double>(T_old, T_old + N) : cs.T;
  cs.T_old_old = T_old_old ? vector<double>(T_old_old, T_old_old + N) : cs.T;
  return 0;
}

int orc_temperature_download(OrcCase* c, double* T, double* gt) {
  const Case& cs = c->cs;
  if (T) std::copy(cs.T.begin(), cs.T.end(), T);
  if (gt) std::copy(cs.gt.begin(), cs.gt.end(), gt);
  return 0;
}

int orc_simple_run(OrcCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier) {
  *ier = simple_run(c->cs, nsteps, log, logcap, nrec);
  return 0;
}

int orc_piso_run(OrcCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier) {
  *ier = piso_run(c->cs, nsteps, log, logcap, nrec);
  return 0;
}

int orc_pimple_run(OrcCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier) {
  *ier = pimple_run(c->cs, nsteps, log, logcap, nrec);
  return 0;
}

// Expose the intermediate objects for element-wise parity checks.
int orc_geometry(OrcCase* c, double* xf, double* sf, double* area, double* vol, double* xc, double* lf) {
  Case& cs = c->cs;
  std::copy(cs.g.xf.begin(), cs.g.xf.end(), xf);
  std::copy(cs.g.sf.begin(), cs.g.sf.end(), sf);
  std::copy(cs.g.area.begin(), cs.g.area.end(), area);
  std::copy(cs.g.vol.begin(), cs.g.vol.end(), vol);
  std::copy(cs.g.xc.begin(), cs.g.xc.end(), xc);
  std::copy(cs.lf.begin(), cs.lf.end(), lf);
  return 0;
}

int orc_connectivity(OrcCase* c, int32_t* cf_ptr, int32_t* cf, int32_t* c2c_ptr, int32_t* c2c, int32_t* row_ptr,
                     int32_t* col_idx, int32_t* nnz) {
  Case& cs = c->cs;
  int N = cs.m.ncells;
  for (int i = 0; i <= N; ++i) {
    cf_ptr[i] = cs.conn.cf_ptr[i] + 1;
    c2c_ptr[i] = cs.conn.c2c_ptr[i] + 1;
    row_ptr[i] = cs.amat.row_ptr[i] + 1;
  }
  for (size_t k = 0; k < cs.conn.cf.size(); ++k) cf[k] = cs.conn.cf[k] + 1;
  for (size_t k = 0; k < cs.conn.c2c.size(); ++k) c2c[k] = cs.conn.c2c[k] + 1;
  for (size_t k = 0; k < cs.amat.col_idx.size(); ++k) col_idx[k] = cs.amat.col_idx[k] + 1;
  *nnz = (int32_t)cs.amat.col_idx.size();
  return 0;
}

// One step of the pipeline, for kernel-level parity: what = 0 gradients,
// 1..3 momentum assembly of component what (returns A.val, rhs, ap),
// 4 Rhie-Chow fluxes, 5 PPE assembly (A.val, rhs), 6 correct_fields with pp.
int orc_stage(OrcCase* c, int what, double* aval, double* rhs, double* ap, const double* pp_in) {
  Case& cs = c->cs;
  if (what == 0) {
    compute_gradients(cs);
  } else if (what >= 1 && what <= 3) {
    momentum_assembly(cs, what - 1);
    if (aval) std::copy(cs.amat.val.begin(), cs.amat.val.end(), aval);
    if (rhs) std::copy(cs.rhs.begin(), cs.rhs.end(), rhs);
    if (ap) std::copy(cs.ap.begin(), cs.ap.end(), ap);
  } else if (what == 4) {
    flux_rhiechow(cs);
  } else if (what == 5) {
    ppe_assembly(cs);
    if (aval) std::copy(cs.pmat.val.begin(), cs.pmat.val.end(), aval);
    if (rhs) std::copy(cs.rhs.begin(), cs.rhs.end(), rhs);
  } else if (what == 6) {
    cs.pp.assign(pp_in, pp_in + cs.m.ncells);
    correct_fields(cs);
  } else if (what == 7) {
    temperature_assembly(cs);
    if (aval) std::copy(cs.amat.val.begin(), cs.amat.val.end(), aval);
    if (rhs) std::copy(cs.rhs.begin(), cs.rhs.end(), rhs);
    if (ap) std::copy(cs.ap.begin(), cs.ap.end(), ap);
  } else {
    return MGPU_E_ARG;
  }
  return 0;
}

int orc_set_apc(OrcCase* c, const double* apc, int ts_order) {
  Case& cs = c->cs;
  if (apc) cs.apc.assign(apc, apc + cs.m.ncells);
  cs.ts_order = ts_order;
  return 0;
}

// set_interface_vel / set_interface_p (mod_uns_bc.f90:730-760): faces 1-based
int orc_interface_set(OrcCase* c, int n, const int32_t* faces, const double* u, const double* p) {
  BC& b = c->cs.bcs;
  for (int k = 0; k < n; ++k) {
    const int i = faces[k] - 1;
    if (i < 0 || i >= c->cs.m.nfaces) return MGPU_E_ARG;
    if (u)
      for (int q = 0; q < 3; ++q) b.iface_vel[3 * (size_t)i + q] = u[3 * (size_t)k + q];
    if (p) b.iface_p[i] = p[k];
  }
  return 0;
}

// set_interface_T / set_interface_q / set_interface_T_mode
// (mod_uns_bc.f90:750-793): faces 1-based
int orc_interface_set_T(OrcCase* c, int n, const int32_t* faces, const double* T, const double* q,
                        const int32_t* mode) {
  BC& b = c->cs.bcs;
  for (int k = 0; k < n; ++k) {
    const int i = faces[k] - 1;
    if (i < 0 || i >= c->cs.m.nfaces) return MGPU_E_ARG;
    if (T) b.iface_T[i] = T[k];
    if (q) b.iface_q[i] = q[k];
    if (mode) b.iface_T_mode[i] = mode[k];
  }
  return 0;
}

// set_iface_p_dirichlet (mod_uns_bc.f90:810-813)
int orc_interface_mode(OrcCase* c, int flag) {
  c->cs.bcs.iface_p_dir = flag != 0;
  return 0;
}

// uns_solver_extract_iface (mod_uns_driver.f90:274-330), fluid owner cells:
// interface groups in order, their faces in face order
int orc_interface_extract(OrcCase* c, int cap, int32_t* faces, double* u, double* p, double* T, int* n) {
  const Case& cs = c->cs;
  int k = 0;
  for (const Group& g : cs.bcs.gb) {
    if (g.btype != MGPU_BC_INTERFACE) continue;
    for (int i : g.faces) {
      if (k < cap) {
        const int c0 = cs.m.c0[i];
        if (faces) faces[k] = i + 1;
        if (u)
          for (int q = 0; q < 3; ++q) u[3 * k + q] = cs.u[3 * c0 + q];
        if (p) p[k] = cs.p[c0];
        if (T) T[k] = cs.T[c0];
      }
      ++k;
    }
  }
  *n = k;
  return 0;
}

int orc_nan_scan(OrcCase* c, int* ifin, int* field, int* cell, double* val, int* kind) {
  *ifin = nan_scan(c->cs, *field, *cell, *val, *kind);
  return 0;
}

// Stand-alone Krylov solve on a 1-based CSR matrix (see mgpu_krylov_solve).
int orc_krylov_solve(int n, const int32_t* row_ptr, const int32_t* col_idx, const double* val, const double* b,
                     double* x, double tol, int maxit, int method, int norm_mode, int* it, double* res, int* ierr) {
  CSR A;
  to_csr(n, row_ptr, col_idx, val, A);
  Norm nrm{norm_mode};
  switch (method) {
    case 0: bicgstab(A, b, x, tol, maxit, *it, *res, *ierr, 0, nrm); break;
    case 1: pcg(A, b, x, tol, maxit, *it, *res, *ierr, 1, nrm); break;
    case 2: pcg(A, b, x, tol, maxit, *it, *res, *ierr, 2, nrm); break;
    case 3: bicgstab(A, b, x, tol, maxit, *it, *res, *ierr, 1, nrm); break;
    case 4: pcg(A, b, x, tol, maxit, *it, *res, *ierr, 0, nrm); break;
    default: return MGPU_E_ARG;
  }
  return 0;
}

int orc_csr_matvec(int n, const int32_t* row_ptr, const int32_t* col_idx, const double* val, const double* x,
                   double* y) {
  CSR A;
  to_csr(n, row_ptr, col_idx, val, A);
  csr_matvec(A, x, y);
  return 0;
}

// Factorisations alone, for element-wise checks of the device factor kernels.
int orc_factor(int n, const int32_t* row_ptr, const int32_t* col_idx, double* val, int kind) {
  CSR A;
  to_csr(n, row_ptr, col_idx, val, A);
  int e = kind == 0 ? ilu0_factor(A) : ic0_factor(A);
  std::copy(A.val.begin(), A.val.end(), val);
  return e;
}

double orc_norm2(const double* a, long n) { return norm2_scaled(a, n); }

}  // extern "C"
