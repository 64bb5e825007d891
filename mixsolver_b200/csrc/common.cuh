// common.cuh -- shared device helpers of the B200 SIMPLE/PISO path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cfloat>
#include <cmath>
#include <string>

#include "../../include/mixgpu.h"

namespace mgpu {

using std::fabs;
using std::fmax;
using std::fmin;
using std::sqrt;

// --- error plumbing -------------------------------------------------------
void set_error(const std::string& msg);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);

#define MGPU_CUDA(call)                                                    \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) return ::mgpu::cuda_fail(e_, #call, __FILE__, __LINE__); \
  } while (0)

#define MGPU_LAUNCH_CHECK(what)                                            \
  do {                                                                     \
    cudaError_t e_ = cudaGetLastError();                                   \
    if (e_ != cudaSuccess) return ::mgpu::cuda_fail(e_, what, __FILE__, __LINE__); \
  } while (0)

constexpr double DTINY = DBL_MIN;  // tiny(1.0_dp)

// gfortran NORM2 of a 3-vector (scaled sum of squares, scale starting at 1).
__host__ __device__ inline double norm3(double a, double b, double c) {
  double result = 0.0, scale = 1.0;
  double v[3] = {a, b, c};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (v[i] != 0.0) {
      double ax = fabs(v[i]);
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
  return scale * sqrt(result);
}

// dot_product of 3-vectors in gfortran's inline order ((0+a1b1)+a2b2)+a3b3.
__host__ __device__ inline double dot3(double a0, double a1, double a2, double b0, double b1, double b2) {
  double s = 0.0;
  s = s + a0 * b0;
  s = s + a1 * b1;
  s = s + a2 * b2;
  return s;
}

// Boundary group as the device sees it (bcgroup_t, mod_uns_bc.f90:80-110).
struct DevGroup {
  int btype;
  int prfl_axis;  // 0-based
  int has_lid;
  int lid_dir;  // 0-based
  double uvel[3];
  double pval;
  double uspeed;
  double prfl_mean, prfl_span, prfl_origin;
  double lid_coord, lid_tol;
  double lid_vel[3];
  // thermal data (walls, outlets, inlets): zone type/values, plane filters
  int ttype, ntbc;
  double tval, qval, tbc_tol;
  int tbc_pdir[4], tbc_ttype[4];  // pdir 0-based
  double tbc_pcoord[4], tbc_tval[4], tbc_qval[4];
};

// Boundary state in effect besides the groups: the cold-start ramp factors and
// the coupling interface (per-face values the peer solver sets, and whether
// the interface is pressure-Dirichlet, mod_uns_bc.f90:28-77).
struct Ramp {
  double inlet, pval;         // g_inlet_ramp_factor, g_pval_ramp_factor
  const double* ivel = nullptr;  // iface_vel, 3 planes of F (interface zones only)
  const double* ip = nullptr;    // iface_p
  long F = 0;
  int ipdir = 0;                 // g_iface_p_dir
  const double* iT = nullptr;    // iface_T (energy cases)
  const double* iq = nullptr;    // iface_q
  const int* itm = nullptr;      // iface_T_mode: 0 Dirichlet, 1 Neumann
};

#ifdef __CUDACC__
// bc_face_vel, mod_uns_bc.f90:400-509
__device__ inline void bc_face_vel(const DevGroup& g, const Ramp& rp, double xf0, double xf1, double xf2,
                                   double s0, double s1, double s2, double u0, double u1, double u2,
                                   double& f0, double& f1, double& f2, long face = -1) {
  double xf[3] = {xf0, xf1, xf2};
  switch (g.btype) {
    case MGPU_BC_INTERFACE:  // the peer's face velocity, or extrapolated when p is the interface constraint
      if (rp.ipdir) {
        f0 = u0;
        f1 = u1;
        f2 = u2;
      } else {
        f0 = rp.ivel[face];
        f1 = rp.ivel[rp.F + face];
        f2 = rp.ivel[2 * rp.F + face];
      }
      return;
    case MGPU_BC_WALL:
      if (g.has_lid && fabs(xf[g.lid_dir] - g.lid_coord) <= g.lid_tol) {
        f0 = g.lid_vel[0];
        f1 = g.lid_vel[1];
        f2 = g.lid_vel[2];
      } else {
        f0 = f1 = f2 = 0.0;
      }
      return;
    case MGPU_BC_SYMMETRY: {
      double ns = norm3(s0, s1, s2);
      double n0 = s0 / ns, n1 = s1 / ns, n2 = s2 / ns;
      double un = dot3(u0, u1, u2, n0, n1, n2);
      f0 = u0 - 2.0 * un * n0;
      f1 = u1 - 2.0 * un * n1;
      f2 = u2 - 2.0 * un * n2;
      return;
    }
    case MGPU_BC_VINLET:
      f0 = g.uvel[0];
      f1 = g.uvel[1];
      f2 = g.uvel[2];
      return;
    case MGPU_BC_VINLET_PARAB: {
      double ns = norm3(s0, s1, s2);
      double n0 = s0 / ns, n1 = s1 / ns, n2 = s2 / ns;
      double xi = (xf[g.prfl_axis] - g.prfl_origin) / g.prfl_span;
      xi = fmax(0.0, fmin(1.0, xi));
      double uspc = 6.0 * g.prfl_mean * xi * (1.0 - xi);
      f0 = -uspc * n0;
      f1 = -uspc * n1;
      f2 = -uspc * n2;
      return;
    }
    case MGPU_BC_MASSINLET: {
      double ns = norm3(s0, s1, s2);
      double n0 = s0 / ns, n1 = s1 / ns, n2 = s2 / ns;
      f0 = -g.uspeed * rp.inlet * n0;
      f1 = -g.uspeed * rp.inlet * n1;
      f2 = -g.uspeed * rp.inlet * n2;
      return;
    }
    case MGPU_BC_FARFIELD: {
      double ns = norm3(s0, s1, s2);
      double n0 = s0 / ns, n1 = s1 / ns, n2 = s2 / ns;
      double un = dot3(g.uvel[0], g.uvel[1], g.uvel[2], n0, n1, n2);
      if (un < 0.0) {
        f0 = g.uvel[0];
        f1 = g.uvel[1];
        f2 = g.uvel[2];
      } else {
        f0 = u0;
        f1 = u1;
        f2 = u2;
      }
      return;
    }
    case MGPU_BC_SLIPWALL: {
      double ns = norm3(s0, s1, s2);
      double n0 = s0 / ns, n1 = s1 / ns, n2 = s2 / ns;
      double un = dot3(u0, u1, u2, n0, n1, n2);
      f0 = u0 - un * n0;
      f1 = u1 - un * n1;
      f2 = u2 - un * n2;
      return;
    }
    default:
      f0 = u0;
      f1 = u1;
      f2 = u2;
  }
}

// bc_face_p, mod_uns_bc.f90:514-549
__device__ inline double bc_face_p(const DevGroup& g, const Ramp& rp, double pP, long face = -1) {
  if (g.btype == MGPU_BC_POUTLET || g.btype == MGPU_BC_FARFIELD) return g.pval * rp.pval;
  if (g.btype == MGPU_BC_INTERFACE && rp.ipdir) return rp.ip[face];
  return pP;
}

// bc_face_T, mod_uns_bc.f90:560-703 (the clear-fluid branch): the face
// temperature and heat flux of a boundary face and whether it is Neumann.
// Interface faces take the peer's temperature, 0 on this path.
__device__ inline void bc_face_T(const DevGroup& g, const Ramp& rp, long face, double xf0, double xf1, double xf2,
                                 double T_cell, double& T_face, double& q_face, bool& neumann) {
  T_face = T_cell;
  q_face = 0.0;
  neumann = true;
  const int bt = g.btype;
  if (bt == MGPU_BC_WALL || bt == MGPU_BC_POUTLET || bt == MGPU_BC_OUTFLOW) {
    int tt = g.ttype;
    double tv = g.tval, qv = g.qval;
    const double xf[3] = {xf0, xf1, xf2};
    for (int ipl = 0; ipl < g.ntbc; ++ipl)
      if (fabs(xf[g.tbc_pdir[ipl]] - g.tbc_pcoord[ipl]) <= g.tbc_tol) {
        tt = g.tbc_ttype[ipl];
        tv = g.tbc_tval[ipl];
        qv = g.tbc_qval[ipl];
        break;
      }
    if (tt == 1) {
      neumann = false;
      T_face = tv;
    } else if (tt == 2) {
      q_face = qv;
    }
  } else if (bt == MGPU_BC_VINLET || bt == MGPU_BC_VINLET_PARAB || bt == MGPU_BC_MASSINLET) {
    neumann = false;
    T_face = g.tval;
  } else if (bt == MGPU_BC_INTERFACE) {  // the peer's temperature, or its heat flux (CHT mode)
    if (rp.itm[face] == 1) {
      q_face = rp.iq[face];
    } else {
      neumann = false;
      T_face = rp.iT[face];
    }
  }
}

// bc_face_p_dirichlet, mod_uns_bc.f90:879-893 (ipdir: g_iface_p_dir); the
// one-rank ppe_assembly_mpi of the transient drivers counts only pressure
// outlets and far fields (mod_uns_simple_mpi.f90:905-907, 944-945): mpi = 1
__device__ inline bool p_dirichlet(int btype, int ipdir = 0, int mpi = 0) {
  return btype == MGPU_BC_POUTLET || btype == MGPU_BC_FARFIELD || (btype == MGPU_BC_INTERFACE && ipdir && !mpi);
}
#endif


inline unsigned ceil_div(long a, long b) { return (unsigned)((a + b - 1) / b); }

}  // namespace mgpu
