// assembly.cu -- face-loop kernels of the SIMPLE/PISO path (FP64 parity form).
//
// The reference accumulates cell sums inside face loops (grad(c0) += ...,
// grad(c1) -= ...). Here every cell gathers its own faces in ascending face
// order through the cell->face lists of build_connectivity, so each cell sum
// sees exactly the same addends in exactly the same order: no atomics, and the
// results are bit-identical to the Fortran loops (compiled without FMA
// contraction). Per-face quantities (Rhie-Chow flux, flux correction) run one
// thread per face.
//
// Reference: src/unstructured/mod_uns_geometry.f90:40-174 (geometry),
// mod_uns_fields.f90:147-157 (lf) and :164-374 (Green-Gauss gradients),
// mod_uns_simple.f90:928-1338 (momentum_assembly), :1346-1408
// (velocity_limiter), :1413-1450 (flux_rhiechow), :1463-1547 (outflow
// scaling), :1552-1644 (ppe_assembly), :1649-1739 (correct_fields),
// :236-247 and :2375-2426 (diagnostics, nan_scan).

#include "assembly.cuh"

namespace mgpu {

extern int g_gather_faces;  // krylov.cu: the gather_faces tuning key

namespace {

// The ramp factors in effect (g_inlet_ramp_factor, g_pval_ramp_factor of
// mod_uns_bc.f90:28-37): kept with the case, 1 until a SIMPLE iteration of a
// run with inlet_ramp > 1 sets them (b_begin_iter), and left at their last
// value afterwards, as the reference's module variables are -- so the
// gradients a run computes before its first iteration see the previous value.
__device__ __forceinline__ Ramp ramp_of(const DeviceCase& d) {
  return Ramp{d.ramp[0],     d.ramp[1],    d.iface_vel, d.iface_p,       (long)d.F,
              d.iface_pdir, d.iface_T,    d.iface_q,   d.iface_tmode};
}
// the interface temperature data alone (bc_face_T reads no ramp factor)
__device__ __forceinline__ Ramp thermal_iface(const DeviceCase& d) {
  Ramp r{1.0, 1.0};
  r.F = d.F;
  r.iT = d.iface_T;
  r.iq = d.iface_q;
  r.itm = d.iface_tmode;
  return r;
}

// ---------------- geometry (setup) ----------------------------------------

// face_props: Newell area vector, area, fan-triangulated centroid
__global__ void k_face_props(int F, const double* __restrict__ x, const int* __restrict__ fptr,
                             const int* __restrict__ fnodes, double* xf, double* sf, double* area) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F) return;
  const int b = fptr[i], n = fptr[i + 1] - b;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int j = 0; j < n; ++j) {
    const int jn = (j + 1) % n;
    const double* p1 = x + 3 * (long)fnodes[b + j];
    const double* p2 = x + 3 * (long)fnodes[b + jn];
    const double c0 = p1[1] * p2[2] - p1[2] * p2[1];
    const double c1 = p1[2] * p2[0] - p1[0] * p2[2];
    const double c2 = p1[0] * p2[1] - p1[1] * p2[0];
    s0 = s0 + 0.5 * c0;
    s1 = s1 + 0.5 * c1;
    s2 = s2 + 0.5 * c2;
  }
  const double a = norm3(s0, s1, s2);
  double e0 = 0.0, e1 = 0.0, e2 = 0.0, at = 0.0;
  const double* p1 = x + 3 * (long)fnodes[b];
  for (int j = 1; j < n - 1; ++j) {
    const double* p2 = x + 3 * (long)fnodes[b + j];
    const double* p3 = x + 3 * (long)fnodes[b + j + 1];
    const double u0 = p2[0] - p1[0], u1 = p2[1] - p1[1], u2 = p2[2] - p1[2];
    const double v0 = p3[0] - p1[0], v1 = p3[1] - p1[1], v2 = p3[2] - p1[2];
    const double t0 = (u1 * v2 - u2 * v1) * 0.5;
    const double t1 = (u2 * v0 - u0 * v2) * 0.5;
    const double t2 = (u0 * v1 - u1 * v0) * 0.5;
    const double ns = norm3(t0, t1, t2);
    e0 = e0 + ns * ((p1[0] + p2[0]) + p3[0]) / 3.0;
    e1 = e1 + ns * ((p1[1] + p2[1]) + p3[1]) / 3.0;
    e2 = e2 + ns * ((p1[2] + p2[2]) + p3[2]) / 3.0;
    at = at + ns;
  }
  if (at > 0.0) {
    e0 = e0 / at;
    e1 = e1 / at;
    e2 = e2 / at;
  }
  xf[i] = e0;
  xf[F + i] = e1;
  xf[2 * F + i] = e2;
  sf[i] = s0;
  sf[F + i] = s1;
  sf[2 * F + i] = s2;
  area[i] = a;
}

// prov_centers: node average of each cell (nodes counted once per face visit)
__global__ void k_prov_centers(int N, const double* __restrict__ x, const int* __restrict__ fptr,
                               const int* __restrict__ fnodes, const int* __restrict__ cf_ptr,
                               const int* __restrict__ cf, double* pcen) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  int cnt = 0;
  for (int k = cf_ptr[c]; k < cf_ptr[c + 1]; ++k) {
    const int f = cf[k];
    for (int j = fptr[f]; j < fptr[f + 1]; ++j) {
      const double* xn = x + 3 * (long)fnodes[j];
      a0 = a0 + xn[0];
      a1 = a1 + xn[1];
      a2 = a2 + xn[2];
      ++cnt;
    }
  }
  if (cnt > 0) {
    a0 = a0 / (double)cnt;
    a1 = a1 / (double)cnt;
    a2 = a2 / (double)cnt;
  }
  pcen[c] = a0;
  pcen[N + c] = a1;
  pcen[2 * N + c] = a2;
}

__global__ void k_orient(int F, int N, const int* __restrict__ c0, const double* __restrict__ xf,
                         const double* __restrict__ pcen, double* sf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F) return;
  const int a = c0[i];
  const double d0 = xf[i] - pcen[a], d1 = xf[F + i] - pcen[N + a], d2 = xf[2 * F + i] - pcen[2 * N + a];
  const double dotv = dot3(sf[i], sf[F + i], sf[2 * F + i], d0, d1, d2);
  if (dotv < 0.0) {
    sf[i] = -sf[i];
    sf[F + i] = -sf[F + i];
    sf[2 * F + i] = -sf[2 * F + i];
  }
}

// pyramid decomposition (accumulate_cell) gathered per cell in face order
__global__ void k_cell_volumes(int N, int F, const int* __restrict__ c0, const int* __restrict__ cf_ptr,
                               const int* __restrict__ cf, const double* __restrict__ xf,
                               const double* __restrict__ sf, const double* __restrict__ pcen, double* vol,
                               double* xc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const double THIRD = 1.0 / 3.0, QRTR = 1.0 / 4.0;
  const double p0 = pcen[c], p1 = pcen[N + c], p2 = pcen[2 * N + c];
  double v = 0.0, x0 = 0.0, x1 = 0.0, x2 = 0.0;
  for (int k = cf_ptr[c]; k < cf_ptr[c + 1]; ++k) {
    const int f = cf[k];
    const double sgn = (c0[f] == c) ? 1.0 : -1.0;
    const double f0 = xf[f], f1 = xf[F + f], f2 = xf[2 * F + f];
    const double dv = THIRD * dot3(sf[f], sf[F + f], sf[2 * F + f], f0 - p0, f1 - p1, f2 - p2) * sgn;
    v = v + dv;
    x0 = x0 + dv * ((1.0 - QRTR) * f0 + QRTR * p0);
    x1 = x1 + dv * ((1.0 - QRTR) * f1 + QRTR * p1);
    x2 = x2 + dv * ((1.0 - QRTR) * f2 + QRTR * p2);
  }
  if (v > 0.0) {
    x0 = x0 / v;
    x1 = x1 / v;
    x2 = x2 / v;
  }
  vol[c] = v;
  xc[c] = x0;
  xc[N + c] = x1;
  xc[2 * N + c] = x2;
}

// Per-face constants: lf (init_fields), |d|, d.S, the momentum diffusion
// coefficient and the non-orthogonal correction vector, each formed with the
// reference's expression so it equals the value recomputed in its face loops.
__global__ void k_face_consts(DeviceCase d, AsmParams P) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int F = d.F, N = d.N;
  if (i >= F) return;
  const int a = d.c0[i], b = d.c1[i];
  const double s0 = d.sf[i], s1 = d.sf[F + i], s2 = d.sf[2 * F + i];
  const double f0 = d.xf[i], f1 = d.xf[F + i], f2 = d.xf[2 * F + i];
  const double area = d.area[i];
  const double POROSITY_FLOOR = 1.0e-8;
  const double mu_eff = P.mu / fmax(1.0, POROSITY_FLOOR);  // pure fluid: porosity 1
  if (b < 0) {
    d.lf[i] = 1.0;
    const double dw = norm3(f0 - d.xc[a], f1 - d.xc[N + a], f2 - d.xc[2 * N + a]);
    d.dn[i] = dw;
    d.Dm[i] = mu_eff * area / dw;
    d.dsf[i] = 0.0;
    d.mnc[i] = 0.0;
    d.tv[i] = d.tv[F + i] = d.tv[2 * F + i] = 0.0;
    return;
  }
  const double d0 = norm3(f0 - d.xc[a], f1 - d.xc[N + a], f2 - d.xc[2 * N + a]);
  const double d1 = norm3(d.xc[b] - f0, d.xc[N + b] - f1, d.xc[2 * N + b] - f2);
  const double lf = d1 / (d0 + d1);
  d.lf[i] = lf;
  const double v0 = d.xc[b] - d.xc[a], v1 = d.xc[N + b] - d.xc[N + a], v2 = d.xc[2 * N + b] - d.xc[2 * N + a];
  const double dn = norm3(v0, v1, v2);
  d.dn[i] = dn;
  d.dsf[i] = dot3(v0, v1, v2, s0, s1, s2);
  const double mu_f = lf * mu_eff + (1.0 - lf) * mu_eff;
  if (P.nonorth_corr > 0.0) {
    const double sd = dot3(s0, s1, s2, v0, v1, v2);
    d.Dm[i] = mu_f * (area * area) / sd;
    const double q = (area * area) / sd;
    d.tv[i] = s0 - v0 * q;
    d.tv[F + i] = s1 - v1 * q;
    d.tv[2 * F + i] = s2 - v2 * q;
  } else {
    d.Dm[i] = mu_f * area / dn;
    d.tv[i] = d.tv[F + i] = d.tv[2 * F + i] = 0.0;
  }
  d.mnc[i] = P.nonorth_corr * mu_f;
}

// ---------------- per-iteration kernels ------------------------------------

// compute_gradients: Green-Gauss gp and gu (gu plane = comp*3 + dir)
// Green-Gauss gradients of p and u (compute_gradients / grad_scalar,
// mod_uns_fields.f90:164-374): one thread per cell, its faces in the cell's
// order. K faces at a time go through three load phases (face indices; face
// data and the other cell; the other cell's values) before any sum, so a
// thread waits about three memory latencies per K faces instead of three per
// face; the sums keep the face order and association (bit-exact for every K).
template <int K = 1>
__device__ __forceinline__ void b_gradients(const DeviceCase& d, const AsmParams& P, const int c) {
  if (d.st->abort || c >= d.N) return;
  const int N = d.N, F = d.F;
  const Ramp rp = ramp_of(d);
  const double *u0 = d.u, *u1 = d.u + N, *u2 = d.u + 2 * N;
  double g[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) g[k] = 0.0;
  const int kb = d.cf_ptr[c], ke = d.cf_ptr[c + 1];
  const double pc = d.p[c], uc0 = u0[c], uc1 = u1[c], uc2 = u2[c];
  for (int k0 = kb; k0 < ke; k0 += K) {
    int fk[K], ok[K];
    bool own[K];
    double lf[K], S0[K], S1[K], S2[K], po[K], w0o[K], w1o[K], w2o[K];
#pragma unroll
    for (int j = 0; j < K; ++j) fk[j] = k0 + j < ke ? d.cf[k0 + j] : -1;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      ok[j] = -1;
      own[j] = true;
      lf[j] = S0[j] = S1[j] = S2[j] = 0.0;
      if (fk[j] >= 0) {
        const int f = fk[j];
        const int a = d.c0[f], b = d.c1[f];
        own[j] = a == c;
        ok[j] = b < 0 ? -1 : (own[j] ? b : a);
        lf[j] = d.lf[f];
        S0[j] = d.sf[f];
        S1[j] = d.sf[F + f];
        S2[j] = d.sf[2 * F + f];
      }
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      po[j] = w0o[j] = w1o[j] = w2o[j] = 0.0;
      if (ok[j] >= 0) {
        po[j] = d.p[ok[j]];
        w0o[j] = u0[ok[j]];
        w1o[j] = u1[ok[j]];
        w2o[j] = u2[ok[j]];
      }
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (fk[j] < 0) break;
      const int f = fk[j];
      double pf, w0, w1, w2;
      if (ok[j] >= 0) {
        // the face's owner (a) and neighbour (b) values, as oriented
        const double l = lf[j], l1 = 1.0 - l;
        const bool o = own[j];
        pf = l * (o ? pc : po[j]) + l1 * (o ? po[j] : pc);
        w0 = l * (o ? uc0 : w0o[j]) + l1 * (o ? w0o[j] : uc0);
        w1 = l * (o ? uc1 : w1o[j]) + l1 * (o ? w1o[j] : uc1);
        w2 = l * (o ? uc2 : w2o[j]) + l1 * (o ? w2o[j] : uc2);
      } else {  // a boundary face: its owner is this cell
        const DevGroup& gr = d.groups[d.fgrp[f]];
        pf = bc_face_p(gr, rp, pc, f);
        bc_face_vel(gr, rp, d.xf[f], d.xf[F + f], d.xf[2 * F + f], S0[j], S1[j], S2[j], uc0, uc1, uc2, w0, w1, w2,
                    f);
      }
      const double phi[4] = {pf, w0, w1, w2};
      if (own[j]) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          g[3 * q + 0] = g[3 * q + 0] + phi[q] * S0[j];
          g[3 * q + 1] = g[3 * q + 1] + phi[q] * S1[j];
          g[3 * q + 2] = g[3 * q + 2] + phi[q] * S2[j];
        }
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          g[3 * q + 0] = g[3 * q + 0] - phi[q] * S0[j];
          g[3 * q + 1] = g[3 * q + 1] - phi[q] * S1[j];
          g[3 * q + 2] = g[3 * q + 2] - phi[q] * S2[j];
        }
      }
    }
  }
  const double v = d.vol[c];
#pragma unroll
  for (int k = 0; k < 3; ++k) d.gp[k * N + c] = g[k] / v;
#pragma unroll
  for (int k = 0; k < 9; ++k) d.gu[k * N + c] = g[3 + k] / v;
}
template <int K>
__global__ void __launch_bounds__(256) k_gradients(DeviceCase d, AsmParams P) {
  b_gradients<K>(d, P, blockIdx.x * blockDim.x + threadIdx.x);
}

// velocity_limiter for one component (Barth-Jespersen psi)
__device__ __forceinline__ void b_limiter(const DeviceCase& d, const AsmParams& P, int comp, const int c) {
  if (d.st->abort || c >= d.N) return;
  const int N = d.N, F = d.F;
  const Ramp rp = ramp_of(d);
  const double* uc_ = d.u + (long)comp * N;
  const double uc = uc_[c];
  double pmin = uc, pmax = uc;
  for (int k = d.cf_ptr[c]; k < d.cf_ptr[c + 1]; ++k) {
    const int f = d.cf[k];
    const int a = d.c0[f], b = d.c1[f];
    if (b >= 0) {
      const double v = uc_[a == c ? b : a];
      pmin = fmin(pmin, v);
      pmax = fmax(pmax, v);
    } else if (d.fgrp[f] >= 0) {
      double w[3];
      bc_face_vel(d.groups[d.fgrp[f]], rp, d.xf[f], d.xf[F + f], d.xf[2 * F + f], d.sf[f], d.sf[F + f],
                  d.sf[2 * F + f], d.u[a], d.u[N + a], d.u[2 * N + a], w[0], w[1], w[2], f);
      pmin = fmin(pmin, w[comp]);
      pmax = fmax(pmax, w[comp]);
    }
  }
  const double g0 = d.gu[(comp * 3 + 0) * N + c], g1 = d.gu[(comp * 3 + 1) * N + c],
               g2 = d.gu[(comp * 3 + 2) * N + c];
  const double x0 = d.xc[c], x1 = d.xc[N + c], x2 = d.xc[2 * N + c];
  double psi = 1.0;
  for (int k = d.cf_ptr[c]; k < d.cf_ptr[c + 1]; ++k) {
    const int f = d.cf[k];
    const double fr = uc + dot3(g0, g1, g2, d.xf[f] - x0, d.xf[F + f] - x1, d.xf[2 * F + f] - x2);
    const double df = fr - uc;
    if (df > 0.0)
      psi = fmin(psi, (pmax - uc) / df);
    else if (df < 0.0)
      psi = fmin(psi, (pmin - uc) / df);
  }
  d.psi[c] = fmax(0.0, fmin(1.0, psi));
}
__global__ void __launch_bounds__(256) k_limiter(DeviceCase d, AsmParams P, int comp) {
  b_limiter(d, P, comp, blockIdx.x * blockDim.x + threadIdx.x);
}

// momentum_assembly (mod_uns_simple.f90:928-1338), the part after the
// interior faces: boundary faces (:1123-1227), sources (:1233-1284), time term
// (:1297-1311) and alpha_u relaxation (:1322-1334) of component comp of cell
// c, continuing the interior sums ap and rhs, then A(diag), rhs and ap out.
// LIST: the boundary faces come from the cell's own boundary-face list (the
// same faces in the same order as the cell's face list, with the interior
// faces and the faces without a group left out); otherwise from its face list.
template <bool LIST>
__device__ __forceinline__ void mom_finish(const DeviceCase& d, const AsmParams& P, const Ramp& rp, int comp,
                                           const int c, double ap, double rhs) {
  const int N = d.N, F = d.F;
  const double *u0 = d.u, *u1 = d.u + N, *u2 = d.u + 2 * N;
  const double* ucomp = d.u + (long)comp * N;
  const double* sfc = d.sf + (long)comp * F;
  double* A = d.aval;
  const int kb = LIST ? d.bf_ptr[c] : d.cf_ptr[c], ke = LIST ? d.bf_ptr[c + 1] : d.cf_ptr[c + 1];
  for (int k = kb; k < ke; ++k) {
    const int f = LIST ? d.bf[k] : d.cf[k];
    if (!LIST) {
      if (d.c1[f] >= 0) continue;
      if (d.fgrp[f] < 0) continue;
    }
    const DevGroup& gr = d.groups[d.fgrp[f]];
    const double s0 = d.sf[f], s1 = d.sf[F + f], s2 = d.sf[2 * F + f];
    double w[3];
    bc_face_vel(gr, rp, d.xf[f], d.xf[F + f], d.xf[2 * F + f], s0, s1, s2, u0[c], u1[c], u2[c], w[0], w[1],
                w[2], f);
    const double pf = bc_face_p(gr, rp, d.p[c], f);
    const double D = d.Dm[f];
    const double Fm = P.rho * dot3(w[0], w[1], w[2], s0, s1, s2);
    switch (gr.btype) {
      case MGPU_BC_WALL:
      case MGPU_BC_SYMMETRY:
      case MGPU_BC_VINLET:
      case MGPU_BC_VINLET_PARAB:
      case MGPU_BC_SLIPWALL:
      case MGPU_BC_MASSINLET:
        ap = ap + D + fmax(Fm, 0.0);
        rhs = rhs + D * w[comp] - Fm * w[comp];
        break;
      case MGPU_BC_POUTLET:
      case MGPU_BC_OUTFLOW:
        ap = ap + fmax(Fm, 0.0);
        rhs = rhs - fmin(Fm, 0.0) * ucomp[c];
        break;
      case MGPU_BC_FARFIELD:
        if (Fm < 0.0) {
          ap = ap + D + fmax(Fm, 0.0);
          rhs = rhs + D * w[comp] - Fm * w[comp];
        } else {
          ap = ap + Fm;
        }
        break;
      case MGPU_BC_INTERFACE:  // mod_uns_simple.f90:1144-1176 (velocity- or pressure-Dirichlet interface)
        if (!rp.ipdir) {
          ap = ap + D + fmax(Fm, 0.0);
          rhs = rhs + D * w[comp] - Fm * w[comp];
        } else {
          ap = ap + fmax(Fm, 0.0);
          rhs = rhs - fmin(Fm, 0.0) * ucomp[c];
        }
        break;
      default:
        break;
    }
    rhs = rhs - pf * sfc[f];
  }
  const double vol = d.vol[c];
  // Boussinesq buoyancy (mod_uns_simple.f90:1229-1240), before the body force
  if (P.boussinesq) rhs = rhs - P.rho * P.beta * (d.T[c] - P.tref) * P.gravity[comp] * vol;
  if (P.has_body_force) rhs = rhs + P.body_force[comp] * vol;
  const int ts = d.st->ts_order;
  if (ts == 1) {
    const double at = P.rho * vol / P.dt;
    ap = ap + at;
    rhs = rhs + at * d.u_old[(long)comp * N + c];
  } else if (ts == 2) {
    const double at = P.rho * vol / (2.0 * P.dt);
    ap = ap + 3.0 * at;
    rhs = rhs + at * (4.0 * d.u_old[(long)comp * N + c] - d.u_old_old[(long)comp * N + c]);
  }
  if (ts > 0 && !P.pimple) {
    A[d.diag[c]] = ap;
  } else {
    A[d.diag[c]] = ap / P.alpha_u;
    rhs = rhs + (1.0 - P.alpha_u) / P.alpha_u * ap * ucomp[c];
  }
  d.rhs[c] = rhs;
  d.ap[c] = ap;
}

// momentum_assembly for component comp: row c of A, rhs(c), ap(c)
__device__ __forceinline__ void b_momentum(const DeviceCase& d, const AsmParams& P, int comp, const int c) {
  if (d.st->abort || c >= d.N) return;
  const int N = d.N, F = d.F;
  const Ramp rp = ramp_of(d);
  const double* sfc = d.sf + (long)comp * F;
  double* A = d.aval;
  double ap = 0.0, rhs = 0.0;
  const int kb = d.cf_ptr[c], ke = d.cf_ptr[c + 1];
  // interior faces; every off-diagonal entry of the row belongs to one of
  // them (the diagonal is written by mom_finish)
  for (int k = kb; k < ke; ++k) {
    const int f = d.cf[k];
    const int b = d.c1[f];
    if (b < 0) continue;
    const int a = d.c0[f];
    const bool own = (a == c);
    const double Fm = d.flux[f];
    const double D = d.Dm[f];
    const int slot = d.cf_slot[k];
    const double off = own ? D + fmax(-Fm, 0.0) : D + fmax(Fm, 0.0);
    ap = own ? ap + fmax(Fm, 0.0) + D : ap + fmax(-Fm, 0.0) + D;
    A[slot] = (d.cf_first[k] ? 0.0 : A[slot]) - off;
    const double lf = d.lf[f], l1 = 1.0 - lf;
    if (P.conv_blend > 0.0) {
      const int cu = (Fm > 0.0) ? a : b;
      const double dcv = d.psi[cu] * dot3(d.gu[(comp * 3 + 0) * N + cu], d.gu[(comp * 3 + 1) * N + cu],
                                          d.gu[(comp * 3 + 2) * N + cu], d.xf[f] - d.xc[cu],
                                          d.xf[F + f] - d.xc[N + cu], d.xf[2 * F + f] - d.xc[2 * N + cu]);
      const double dc = P.conv_blend * Fm * dcv;
      rhs = own ? rhs - dc : rhs + dc;
    }
    if (P.nonorth_corr > 0.0) {
      const double gf0 = lf * d.gu[(comp * 3 + 0) * N + a] + l1 * d.gu[(comp * 3 + 0) * N + b];
      const double gf1 = lf * d.gu[(comp * 3 + 1) * N + a] + l1 * d.gu[(comp * 3 + 1) * N + b];
      const double gf2 = lf * d.gu[(comp * 3 + 2) * N + a] + l1 * d.gu[(comp * 3 + 2) * N + b];
      const double noc = d.mnc[f] * dot3(gf0, gf1, gf2, d.tv[f], d.tv[F + f], d.tv[2 * F + f]);
      rhs = own ? rhs + noc : rhs - noc;
    }
    const double pf = lf * d.p[a] + l1 * d.p[b];
    const double S = sfc[f];
    rhs = own ? rhs - pf * S : rhs + pf * S;
  }
  mom_finish<false>(d, P, rp, comp, c, ap, rhs);
}
__global__ void __launch_bounds__(256) k_momentum(DeviceCase d, AsmParams P, int comp) {
  b_momentum(d, P, comp, blockIdx.x * blockDim.x + threadIdx.x);
}

// The interior faces of momentum_assembly (mod_uns_simple.f90:974-1120) for
// all three components at once, without the deferred convection correction
// (conv_blend = 0: the only input that changes between the components' solves
// inside the interior loop is then absent). The matrix row (off-diagonals) and
// ap are the same for every component; the three rhs sums are kept apart, each
// receiving its component's terms in the reference's order. Out: the row of A,
// mom_ap(c), mom_rhs(comp, c); mom_finish<true> completes each component after
// the previous component's solve. K faces' loads at a time (as b_gradients);
// NO: the non-orthogonal correction is on.
template <int K = 1, bool NO = true>
__device__ __forceinline__ void b_mom_interior(const DeviceCase& d, const AsmParams& P, const int c) {
  if (d.st->abort || c >= d.N) return;
  const int N = d.N, F = d.F;
  double* A = d.aval;
  double ap = 0.0, r0 = 0.0, r1 = 0.0, r2 = 0.0;
  const int kb = d.cf_ptr[c], ke = d.cf_ptr[c + 1];
  const bool nonorth = NO && P.nonorth_corr > 0.0;
  const double pc = d.p[c];
  // the cell's own gradient, read once (K = 1: at each face, as the loads
  // then overlap nothing anyway)
  double guc[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) guc[q] = (nonorth && K > 1) ? d.gu[q * N + c] : 0.0;
  // every off-diagonal entry of the row belongs to an interior face: written
  // at its first face, added to at a later one (0 - x is the reference's sum
  // from its zeroed row); the diagonal is written by mom_finish
  for (int k0 = kb; k0 < ke; k0 += K) {
    int fk[K], ok[K], slot[K];
    bool own[K], first[K];
    double Fm[K], Dm[K], lf[K], S0[K], S1[K], S2[K], po[K];
    double tv0[K], tv1[K], tv2[K], mn[K], guo[K][9];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      fk[j] = k0 + j < ke ? d.cf[k0 + j] : -1;
      slot[j] = k0 + j < ke ? d.cf_slot[k0 + j] : -1;
      first[j] = k0 + j < ke ? d.cf_first[k0 + j] != 0 : false;
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      ok[j] = -1;
      own[j] = true;
      Fm[j] = Dm[j] = lf[j] = S0[j] = S1[j] = S2[j] = 0.0;
      tv0[j] = tv1[j] = tv2[j] = mn[j] = 0.0;
      if (fk[j] >= 0) {
        const int f = fk[j];
        const int a = d.c0[f], b = d.c1[f];
        own[j] = a == c;
        ok[j] = b < 0 ? -1 : (own[j] ? b : a);
        if (b >= 0) {
          Fm[j] = d.flux[f];
          Dm[j] = d.Dm[f];
          lf[j] = d.lf[f];
          S0[j] = d.sf[f];
          S1[j] = d.sf[F + f];
          S2[j] = d.sf[2 * F + f];
          if (nonorth) {
            tv0[j] = d.tv[f];
            tv1[j] = d.tv[F + f];
            tv2[j] = d.tv[2 * F + f];
            mn[j] = d.mnc[f];
          }
        }
      }
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      po[j] = ok[j] >= 0 ? d.p[ok[j]] : 0.0;
#pragma unroll
      for (int q = 0; q < 9; ++q) guo[j][q] = (nonorth && ok[j] >= 0) ? d.gu[q * N + ok[j]] : 0.0;
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (fk[j] < 0) break;
      if (ok[j] < 0) continue;
      const bool own_ = own[j];
      const double off = own_ ? Dm[j] + fmax(-Fm[j], 0.0) : Dm[j] + fmax(Fm[j], 0.0);
      ap = own_ ? ap + fmax(Fm[j], 0.0) + Dm[j] : ap + fmax(-Fm[j], 0.0) + Dm[j];
      A[slot[j]] = (first[j] ? 0.0 : A[slot[j]]) - off;
      const double l = lf[j], l1 = 1.0 - l;
      if (nonorth) {
        double nc[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          // gradient components at the owner (a) and neighbour (b), as oriented
          double gc[3];
#pragma unroll
          for (int r = 0; r < 3; ++r) gc[r] = K > 1 ? guc[q * 3 + r] : d.gu[(q * 3 + r) * N + c];
          const double a0 = own_ ? gc[0] : guo[j][q * 3 + 0], b0 = own_ ? guo[j][q * 3 + 0] : gc[0];
          const double a1 = own_ ? gc[1] : guo[j][q * 3 + 1], b1 = own_ ? guo[j][q * 3 + 1] : gc[1];
          const double a2 = own_ ? gc[2] : guo[j][q * 3 + 2], b2 = own_ ? guo[j][q * 3 + 2] : gc[2];
          const double gf0 = l * a0 + l1 * b0;
          const double gf1 = l * a1 + l1 * b1;
          const double gf2 = l * a2 + l1 * b2;
          nc[q] = mn[j] * dot3(gf0, gf1, gf2, tv0[j], tv1[j], tv2[j]);
        }
        r0 = own_ ? r0 + nc[0] : r0 - nc[0];
        r1 = own_ ? r1 + nc[1] : r1 - nc[1];
        r2 = own_ ? r2 + nc[2] : r2 - nc[2];
      }
      const double pf = l * (own_ ? pc : po[j]) + l1 * (own_ ? po[j] : pc);
      r0 = own_ ? r0 - pf * S0[j] : r0 + pf * S0[j];
      r1 = own_ ? r1 - pf * S1[j] : r1 + pf * S1[j];
      r2 = own_ ? r2 - pf * S2[j] : r2 + pf * S2[j];
    }
  }
  d.mom_ap[c] = ap;
  d.mom_rhs[c] = r0;
  d.mom_rhs[N + c] = r1;
  d.mom_rhs[2 * N + c] = r2;
}
template <int K, bool NO>
__global__ void __launch_bounds__(256) k_mom_interior(DeviceCase d, AsmParams P) {
  b_mom_interior<K, NO>(d, P, blockIdx.x * blockDim.x + threadIdx.x);
}

__device__ __forceinline__ void b_mom_finish(const DeviceCase& d, const AsmParams& P, int comp, const int c) {
  if (d.st->abort || c >= d.N) return;
  mom_finish<true>(d, P, ramp_of(d), comp, c, d.mom_ap[c], d.mom_rhs[(long)comp * d.N + c]);
}
__global__ void __launch_bounds__(256) k_mom_finish(DeviceCase d, AsmParams P, int comp) {
  b_mom_finish(d, P, comp, blockIdx.x * blockDim.x + threadIdx.x);
}

__device__ __forceinline__ void b_apc(const DeviceCase& d, double div, const int c) {
  if (d.st->abort || c >= d.N) return;
  d.apc[c] = (div == 1.0) ? d.ap[c] : d.ap[c] / div;
}
__global__ void k_apc(DeviceCase d, double div) { b_apc(d, div, blockIdx.x * blockDim.x + threadIdx.x); }

__global__ void k_fill(double* a, long n, double v) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) a[i] = v;
}

// flux_rhiechow: one thread per face
__device__ __forceinline__ void b_rhiechow(const DeviceCase& d, const AsmParams& P, const int f) {
  if (d.st->abort || f >= d.F) return;
  const int N = d.N, F = d.F;
  const int a = d.c0[f], b = d.c1[f];
  const double s0 = d.sf[f], s1 = d.sf[F + f], s2 = d.sf[2 * F + f];
  if (b < 0) {
    const Ramp rp = ramp_of(d);
    double w0, w1, w2;
    bc_face_vel(d.groups[d.fgrp[f]], rp, d.xf[f], d.xf[F + f], d.xf[2 * F + f], s0, s1, s2, d.u[a], d.u[N + a],
                d.u[2 * N + a], w0, w1, w2, f);
    d.flux[f] = P.rho * dot3(w0, w1, w2, s0, s1, s2);
    return;
  }
  const double lf = d.lf[f], l1 = 1.0 - lf;
  const double uf0 = lf * d.u[a] + l1 * d.u[b];
  const double uf1 = lf * d.u[N + a] + l1 * d.u[N + b];
  const double uf2 = lf * d.u[2 * N + a] + l1 * d.u[2 * N + b];
  const double gp0 = lf * d.gp[a] + l1 * d.gp[b];
  const double gp1 = lf * d.gp[N + a] + l1 * d.gp[N + b];
  const double gp2 = lf * d.gp[2 * N + a] + l1 * d.gp[2 * N + b];
  const double dn = d.dn[f];
  const double pfgrad_n = (d.p[b] - d.p[a]) / dn;
  const double dbf = lf * d.vol[a] / d.apc[a] + l1 * d.vol[b] / d.apc[b];
  d.flux[f] = P.rho * (dot3(uf0, uf1, uf2, s0, s1, s2) +
                       dbf * (dot3(gp0, gp1, gp2, s0, s1, s2) - pfgrad_n * d.dsf[f] / dn));
}
__global__ void __launch_bounds__(256) k_rhiechow(DeviceCase d, AsmParams P) {
  b_rhiechow(d, P, blockIdx.x * blockDim.x + threadIdx.x);
}

// outflow_mass_sums + outflow_mass_scale (mod_uns_simple.f90:1463-1547). The
// reference forms its three sums sequentially in face order, and only that
// order gives its rounding, so each sum stays one dependent chain -- but over
// a compact list of just its own faces in face order (built once per case:
// of_req the fixed-flux boundary faces, of_out the outflow faces), the three
// chains in three threads side by side. The scaling then runs over the
// outflow faces on every thread of the block. Called by all threads of one
// block; only cases with an outflow zone launch it.
__device__ void b_outflow(const DeviceCase& d) {
  __shared__ double s_sum[3];
  if (d.st->abort) return;  // the same for every thread of the block
  const int t = threadIdx.x;
  if (t < 3) {
    double acc = 0.0;
    if (t == 0) {
#pragma unroll 8
      for (int k = 0; k < d.n_of_req; ++k) acc = acc - d.flux[d.of_req[k]];
    } else if (t == 1) {
#pragma unroll 8
      for (int k = 0; k < d.n_of_out; ++k) acc = acc + d.flux[d.of_out[k]];
    } else {
#pragma unroll 8
      for (int k = 0; k < d.n_of_out; ++k) acc = acc + d.area[d.of_out[k]];
    }
    s_sum[t] = acc;
  }
  __syncthreads();
  const double m_req = s_sum[0], m_out = s_sum[1], area_out = s_sum[2];
  if (area_out <= 0.0 || m_req <= 0.0) return;
  const bool scaled = m_out > 1.0e-2 * m_req;
  const double beta = scaled ? m_req / m_out : 0.0;
  for (int k = t; k < d.n_of_out; k += blockDim.x) {
    const int i = d.of_out[k];
    d.flux[i] = scaled ? beta * d.flux[i] : m_req * d.area[i] / area_out;
  }
}
__global__ void k_outflow(DeviceCase d) { b_outflow(d); }

// ppe_assembly: row c of the pressure-correction matrix, rhs(c), pin, pp := 0
// The pressure-correction row of a cell (ppe_assembly, mod_uns_simple.f90:
// 1552-1644), its faces in order, K faces' loads at a time (as b_gradients).
template <int K = 1>
__device__ __forceinline__ void b_ppe(const DeviceCase& d, const AsmParams& P, const int c) {
  if (d.st->abort || c >= d.N) return;
  double* A = d.pval;
  const int rb = d.row_ptr[c], re = d.row_ptr[c + 1], dg = d.diag[c];
  // the diagonal sums in a register in the reference's face order; each
  // off-diagonal entry is written at its first face (0 - af: the reference's
  // zeroed row) and added to at a later one
  double adg = 0.0;
  double rhs = 0.0;
  const int kb = d.cf_ptr[c], ke = d.cf_ptr[c + 1];
  const double volc = d.vol[c], apcc = d.apc[c];
  for (int k0 = kb; k0 < ke; k0 += K) {
    int fk[K], ok[K], slot[K];
    bool own[K], first[K];
    double lf[K], ar[K], dn[K], fl[K], volo[K], apco[K];
#pragma unroll
    for (int j = 0; j < K; ++j) {
      fk[j] = k0 + j < ke ? d.cf[k0 + j] : -1;
      slot[j] = k0 + j < ke ? d.cf_slot[k0 + j] : -1;
      first[j] = k0 + j < ke ? d.cf_first[k0 + j] != 0 : false;
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      ok[j] = -1;
      own[j] = true;
      lf[j] = ar[j] = dn[j] = fl[j] = 0.0;
      if (fk[j] >= 0) {
        const int f = fk[j];
        const int a = d.c0[f], b = d.c1[f];
        own[j] = a == c;
        ok[j] = b < 0 ? -1 : (own[j] ? b : a);
        lf[j] = d.lf[f];
        ar[j] = d.area[f];
        dn[j] = d.dn[f];
        fl[j] = d.flux[f];
      }
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      volo[j] = ok[j] >= 0 ? d.vol[ok[j]] : 0.0;
      apco[j] = ok[j] >= 0 ? d.apc[ok[j]] : 1.0;
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (fk[j] < 0) break;
      const int f = fk[j];
      if (ok[j] < 0) {
        const int gi = d.fgrp[f];
        // af of a pressure-Dirichlet face (the serial rule, which the flux
        // correction uses in every driver); it enters the matrix under the
        // driver's own rule (the transient drivers' ppe_assembly_mpi leaves
        // interface faces out)
        if (gi >= 0 && p_dirichlet(d.groups[gi].btype, d.iface_pdir)) {
          const double dbf = volc / apcc;
          const double af = P.rho * dbf * ar[j] / dn[j];
          if (p_dirichlet(d.groups[gi].btype, d.iface_pdir, d.st->ts_order > 0)) adg = adg + af;
          d.af[f] = af;
        }
        rhs = rhs - fl[j];
        continue;
      }
      const bool o = own[j];
      // the owner (a) and neighbour (b) terms, as the face orients them
      const double va = o ? volc : volo[j], pa = o ? apcc : apco[j];
      const double vb = o ? volo[j] : volc, pb = o ? apco[j] : apcc;
      const double dbf = lf[j] * va / pa + (1.0 - lf[j]) * vb / pb;
      const double af = P.rho * dbf * ar[j] / dn[j];
      adg = adg + af;
      A[slot[j]] = (first[j] ? 0.0 : A[slot[j]]) - af;
      if (o) {
        rhs = rhs - fl[j];
        d.af[f] = af;
      } else {
        rhs = rhs + fl[j];
      }
    }
  }
  A[dg] = adg;
  // the pin of cell 1 when no face is pressure-Dirichlet (serial rule for
  // SIMPLE, the one-rank mpi rule for the transient drivers)
  if (!(P.has_pdir || (d.iface_pdir && d.n_iface > 0 && d.st->ts_order == 0))) {
    if (c == 0) {
      for (int k = rb; k < re; ++k) A[k] = (d.col[k] == 0) ? 1.0 : 0.0;
      rhs = 0.0;
    } else if (d.col[rb] == 0) {
      A[rb] = 0.0;
    }
  }
  d.rhs[c] = rhs;
  d.pp[c] = 0.0;
}
template <int K>
__global__ void __launch_bounds__(256) k_ppe(DeviceCase d, AsmParams P) {
  b_ppe<K>(d, P, blockIdx.x * blockDim.x + threadIdx.x);
}

// correct_fields, cell part: Green-Gauss grad(p') and the u, p updates
// The velocity and pressure correction of a cell (correct_fields,
// mod_uns_simple.f90:1649-1739): the Green-Gauss gradient of p' over its faces
// in order, K faces' loads at a time (as b_gradients).
template <int K = 1>
__device__ __forceinline__ void b_correct_cells(const DeviceCase& d, const AsmParams& P, const int c) {
  if (d.st->abort || c >= d.N) return;
  const int N = d.N, F = d.F;
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  const int kb = d.cf_ptr[c], ke = d.cf_ptr[c + 1];
  const double ppc = d.pp[c];
  for (int k0 = kb; k0 < ke; k0 += K) {
    int fk[K], ok[K];
    bool own[K];
    double lf[K], S0[K], S1[K], S2[K], ppo[K];
#pragma unroll
    for (int j = 0; j < K; ++j) fk[j] = k0 + j < ke ? d.cf[k0 + j] : -1;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      ok[j] = -1;
      own[j] = true;
      lf[j] = S0[j] = S1[j] = S2[j] = 0.0;
      if (fk[j] >= 0) {
        const int f = fk[j];
        const int a = d.c0[f], b = d.c1[f];
        own[j] = a == c;
        ok[j] = b < 0 ? -1 : (own[j] ? b : a);
        lf[j] = d.lf[f];
        S0[j] = d.sf[f];
        S1[j] = d.sf[F + f];
        S2[j] = d.sf[2 * F + f];
      }
    }
#pragma unroll
    for (int j = 0; j < K; ++j) ppo[j] = ok[j] >= 0 ? d.pp[ok[j]] : 0.0;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (fk[j] < 0) break;
      double phif;
      if (ok[j] >= 0) {
        const bool o = own[j];
        phif = lf[j] * (o ? ppc : ppo[j]) + (1.0 - lf[j]) * (o ? ppo[j] : ppc);
      } else {
        const int gi = d.fgrp[fk[j]];
        phif = (gi >= 0 && p_dirichlet(d.groups[gi].btype, d.iface_pdir)) ? 0.0 : ppc;
      }
      if (own[j]) {
        g0 = g0 + phif * S0[j];
        g1 = g1 + phif * S1[j];
        g2 = g2 + phif * S2[j];
      } else {
        g0 = g0 - phif * S0[j];
        g1 = g1 - phif * S1[j];
        g2 = g2 - phif * S2[j];
      }
    }
  }
  const double vol = d.vol[c];
  g0 = g0 / vol;
  g1 = g1 / vol;
  g2 = g2 / vol;
  const double va = vol / d.apc[c];
  d.u[c] = d.u[c] - va * g0;
  d.u[N + c] = d.u[N + c] - va * g1;
  d.u[2 * N + c] = d.u[2 * N + c] - va * g2;
  d.p[c] = (d.st->ts_order > 0) ? d.p[c] + ppc : d.p[c] + P.alpha_p * ppc;
}
template <int K>
__global__ void __launch_bounds__(256) k_correct_cells(DeviceCase d, AsmParams P) {
  b_correct_cells<K>(d, P, blockIdx.x * blockDim.x + threadIdx.x);
}

// correct_fields, flux part
__device__ __forceinline__ void b_correct_flux(const DeviceCase& d, const int f) {
  if (d.st->abort || f >= d.F) return;
  const int a = d.c0[f], b = d.c1[f];
  if (b < 0) {
    const int gi = d.fgrp[f];
    if (gi >= 0 && p_dirichlet(d.groups[gi].btype, d.iface_pdir)) d.flux[f] = d.flux[f] + d.af[f] * d.pp[a];
    return;
  }
  d.flux[f] = d.flux[f] - d.af[f] * (d.pp[b] - d.pp[a]);
}
__global__ void k_correct_flux(DeviceCase d) { b_correct_flux(d, blockIdx.x * blockDim.x + threadIdx.x); }

__device__ __forceinline__ void atomic_max_pos(unsigned long long* a, double v) {
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// Diagnostics of one outer iteration / step: max|imbalance|, max|du|,
// max|u| (transient), max|T - T before its solve| (energy), first non-finite
// value (min over cell*5+field, fields u, v, w, p, T).
__device__ __forceinline__ void b_diag(const DeviceCase& d, int transient, const int c) {
  if (d.st->abort) return;
  double im = 0.0, du = 0.0, um = 0.0, dT = 0.0;
  unsigned long long key = ~0ull;
  if (c < d.N) {
    const int N = d.N;
    for (int k = d.cf_ptr[c]; k < d.cf_ptr[c + 1]; ++k) {
      const int f = d.cf[k];
      im = (d.c0[f] == c) ? im + d.flux[f] : im - d.flux[f];
    }
    im = fabs(im);
    const double* ref = transient ? d.u_old : d.uo;
    const double v[5] = {d.u[c], d.u[N + c], d.u[2 * N + c], d.p[c], d.T[c]};
#pragma unroll
    for (int q = 0; q < 3; ++q) du = fmax(du, fabs(v[q] - ref[(long)q * N + c]));
    if (transient) um = norm3(v[0], v[1], v[2]);
    if (d.energy) dT = fabs(v[4] - d.Tprev[c]);
#pragma unroll
    for (int q = 4; q >= 0; --q)
      if (!isfinite(v[q])) key = (unsigned long long)c * 5ull + (unsigned long long)q;
    if (isnan(im)) im = 0.0;  // a non-finite field is reported by the scan
    if (isnan(du)) du = 0.0;
    if (isnan(um)) um = 0.0;
    if (isnan(dT)) dT = 0.0;
  }
  // warp-level max (exact, order-independent) before the atomics
  for (int o = 16; o > 0; o >>= 1) {
    im = fmax(im, __shfl_xor_sync(0xffffffffu, im, o));
    du = fmax(du, __shfl_xor_sync(0xffffffffu, du, o));
    um = fmax(um, __shfl_xor_sync(0xffffffffu, um, o));
    dT = fmax(dT, __shfl_xor_sync(0xffffffffu, dT, o));
    unsigned long long ko = __shfl_xor_sync(0xffffffffu, key, o);
    key = ko < key ? ko : key;
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(&d.st->imbal_bits, im);
    atomic_max_pos(&d.st->du_bits, du);
    if (transient) atomic_max_pos(&d.st->umax_bits, um);
    if (d.energy) atomic_max_pos(&d.st->dT_bits, dT);
    if (key != ~0ull) atomicMin(&d.st->nan_key, key);
  }
}
__global__ void __launch_bounds__(256) k_diag(DeviceCase d, int transient) {
  b_diag(d, transient, blockIdx.x * blockDim.x + threadIdx.x);
}

// Close the iteration: record, NaN guard (ier 60), convergence, advance.
__device__ void b_diag_finalize(const DeviceCase& d, const AsmParams& P, int transient) {
  DevStatus* st = d.st;
  if (st->abort) return;
  MgpuIterRec* rec = d.recs + st->cur_it;
  if (st->nan_key != ~0ull) {
    const unsigned long long k = st->nan_key;
    const int cell = (int)(k / 5ull), q = (int)(k % 5ull);
    const double v = q < 3 ? d.u[(long)q * d.N + cell] : q == 3 ? d.p[cell] : d.T[cell];
    st->nan_field = q + 1;
    st->nan_cell = cell + 1;
    st->nan_val = v;
    st->nan_kind = isnan(v) ? 1 : 2;
    st->ier = 60;
    st->abort = 1;
    return;
  }
  const double imbal = __longlong_as_double((long long)st->imbal_bits) / P.flux_ref;
  double du = __longlong_as_double((long long)st->du_bits);
  // itl_max and ressum continue over the earlier outer iterations of a PIMPLE
  // step (0 otherwise), as the reference sums them in solve order
  int itl_max = st->acc_itl;
  double ressum = st->acc_res;
  for (int s = 0; s < rec->nsolve && s < MGPU_MAXSOLVE; ++s) itl_max = max(itl_max, rec->lin_it[s]);
  for (int s = 0; s < 3; ++s) ressum = ressum + rec->lin_res[s];
  st->acc_itl = 0;
  st->acc_res = 0.0;
  rec->it = st->cur_it + 1;
  rec->itl_max = itl_max;
  rec->ressum = ressum;
  rec->imbal = imbal;
  const double dTm = d.energy ? __longlong_as_double((long long)st->dT_bits) : 0.0;
  rec->dT_max = dTm;
  if (transient) {
    st->t_now = st->t_now + P.dt;
    du = du / P.dt;
    const double umax = __longlong_as_double((long long)st->umax_bits);
    rec->umax = umax;
    rec->cfl_max = umax * P.dt / P.min_cbrt_vol;
    rec->t_now = st->t_now;
  }
  rec->du_max = du;
  st->imbal_bits = st->du_bits = st->umax_bits = st->dT_bits = 0ull;
  st->cur_it = st->cur_it + 1;
  if (!transient && imbal < P.outer_tol && du < P.outer_tol && dTm < P.outer_tol) {
    st->converged = 1;
    st->abort = 1;
  }
  if (st->it_limit > 0 && st->cur_it >= st->it_limit) st->abort = 1;
}
__global__ void k_diag_finalize(DeviceCase d, AsmParams P, int transient) { b_diag_finalize(d, P, transient); }

// End of a PIMPLE outer iteration that is not the step's last: its solves'
// counts and momentum residuals join the step's running itl_max and ressum
// (the record's slots are reused by the next outer iteration).
__global__ void k_outer_accum(DeviceCase d) {
  DevStatus* st = d.st;
  if (st->abort) return;
  const MgpuIterRec* rec = d.recs + st->cur_it;
  int m = st->acc_itl;
  for (int s = 0; s < rec->nsolve && s < MGPU_MAXSOLVE; ++s) m = max(m, rec->lin_it[s]);
  double r = st->acc_res;
  for (int s = 0; s < 3; ++s) r = r + rec->lin_res[s];
  st->acc_itl = m;
  st->acc_res = r;
}

// SIMPLE: uo := u ; PISO: history shift and time-scheme order
__device__ __forceinline__ void b_begin_iter(const DeviceCase& d, int transient, int time_scheme, int inlet_ramp,
                                             const long i) {
  if (d.st->abort) return;
  const long n3 = 3l * d.N;
  if (i < n3) {
    if (transient) {
      d.u_old_old[i] = d.u_old[i];
      d.u_old[i] = d.u[i];
    } else {
      d.uo[i] = d.u[i];
    }
  }
  if (transient && d.energy && i < d.N) {
    d.T_old_old[i] = d.T_old[i];
    d.T_old[i] = d.T[i];
  }
  if (i == 0) {
    MgpuIterRec* rec = d.recs + d.st->cur_it;
    rec->nsolve = 0;
    if (transient) d.st->ts_order = (d.st->cur_it == 0 || time_scheme == 1) ? 1 : 2;
    // the cold-start ramp of simple_run (mod_uns_simple.f90:150-155): it / inlet_ramp, clamped to [0, 1]
    if (!transient && inlet_ramp > 1) {
      const double f = fmax(0.0, fmin(1.0, (double)(d.st->cur_it + 1) / (double)inlet_ramp));
      d.ramp[0] = f;
      d.ramp[1] = f;
    }
  }
}
__global__ void k_begin_iter(DeviceCase d, int transient, int time_scheme, int inlet_ramp) {
  b_begin_iter(d, transient, time_scheme, inlet_ramp, blockIdx.x * (long)blockDim.x + threadIdx.x);
}

// ---------------- energy equation ------------------------------------------

// The temperature gradient gt (compute_gradients, mod_uns_fields.f90:219-237):
// Green-Gauss over the face values (interior: linear interpolation; boundary:
// bc_face_T's face temperature) in the cell's face order, as k_gradients.
__device__ __forceinline__ void b_tgrad(const DeviceCase& d, const int c) {
  if (d.st->abort || c >= d.N) return;
  const int N = d.N, F = d.F;
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  for (int k = d.cf_ptr[c]; k < d.cf_ptr[c + 1]; ++k) {
    const int f = d.cf[k];
    const int a = d.c0[f], b = d.c1[f];
    double phi;
    if (b >= 0) {
      const double lf = d.lf[f];
      phi = lf * d.T[a] + (1.0 - lf) * d.T[b];
    } else {
      double qf;
      bool neu;
      bc_face_T(d.groups[d.fgrp[f]], thermal_iface(d), f, d.xf[f], d.xf[F + f], d.xf[2 * F + f], d.T[a], phi, qf,
                neu);
    }
    const double s0 = d.sf[f], s1 = d.sf[F + f], s2 = d.sf[2 * F + f];
    if (a == c) {
      g0 = g0 + phi * s0;
      g1 = g1 + phi * s1;
      g2 = g2 + phi * s2;
    } else {
      g0 = g0 - phi * s0;
      g1 = g1 - phi * s1;
      g2 = g2 - phi * s2;
    }
  }
  const double v = d.vol[c];
  d.gt[c] = g0 / v;
  d.gt[N + c] = g1 / v;
  d.gt[2 * N + c] = g2 / v;
}
__global__ void __launch_bounds__(256) k_tgrad(DeviceCase d) { b_tgrad(d, blockIdx.x * blockDim.x + threadIdx.x); }

// temperature_limiter, mod_uns_simple.f90:2302-2361: Barth-Jespersen psi_T
// from the neighbour and boundary-face temperatures (min / max are exact in
// any order)
__device__ __forceinline__ void b_tlimiter(const DeviceCase& d, const int c) {
  if (d.st->abort || c >= d.N) return;
  const int N = d.N, F = d.F;
  const double tc = d.T[c];
  double pmin = tc, pmax = tc;
  for (int k = d.cf_ptr[c]; k < d.cf_ptr[c + 1]; ++k) {
    const int f = d.cf[k];
    const int a = d.c0[f], b = d.c1[f];
    double v;
    if (b >= 0) {
      v = d.T[a == c ? b : a];
    } else {
      double qf;
      bool neu;
      bc_face_T(d.groups[d.fgrp[f]], thermal_iface(d), f, d.xf[f], d.xf[F + f], d.xf[2 * F + f], tc, v, qf, neu);
    }
    pmin = fmin(pmin, v);
    pmax = fmax(pmax, v);
  }
  const double g0 = d.gt[c], g1 = d.gt[N + c], g2 = d.gt[2 * N + c];
  const double x0 = d.xc[c], x1 = d.xc[N + c], x2 = d.xc[2 * N + c];
  double psi = 1.0;
  for (int k = d.cf_ptr[c]; k < d.cf_ptr[c + 1]; ++k) {
    const int f = d.cf[k];
    const double fr = tc + dot3(g0, g1, g2, d.xf[f] - x0, d.xf[F + f] - x1, d.xf[2 * F + f] - x2);
    const double df = fr - tc;
    if (df > 0.0)
      psi = fmin(psi, (pmax - tc) / df);
    else if (df < 0.0)
      psi = fmin(psi, (pmin - tc) / df);
  }
  d.psiT[c] = fmax(0.0, fmin(1.0, psi));
}
__global__ void __launch_bounds__(256) k_tlimiter(DeviceCase d) { b_tlimiter(d, blockIdx.x * blockDim.x + threadIdx.x); }

// temperature_assembly, mod_uns_simple.f90:1748-2037, the clear-fluid
// branch (porosity 1, no porous or solid zones, LTE): k_eff = 1 k + (1 - 1) 0
// and the dispersion terms add 0, formed with the reference's expressions.
// Row c of A (the momentum matrix's storage), rhs(c) and ap(c) (unrelaxed):
// the interior faces in the cell's face order, then its boundary faces, the
// time term and the relaxation, each in the reference's order of sums. The
// interior geometry reuses the face constants (dn, sf.d, and sf - d
// area^2/sf.d, the non-orthogonal vector) that equal the reference's
// per-face expressions.
__device__ __forceinline__ void b_temperature(const DeviceCase& d, const AsmParams& P, const int c) {
  if (d.st->abort || c >= d.N) return;
  const int N = d.N, F = d.F;
  double* A = d.aval;
  const double k_eff = 1.0 * P.k_cond + (1.0 - 1.0) * 0.0;
  double ap = 0.0, rhs = 0.0;
  const int kb = d.cf_ptr[c], ke = d.cf_ptr[c + 1];
  for (int k = kb; k < ke; ++k) {
    const int f = d.cf[k];
    const int b = d.c1[f];
    if (b < 0) continue;
    const int a = d.c0[f];
    const bool own = (a == c);
    const double FT = P.cp * d.flux[f];
    const double lf = d.lf[f];
    double kf = lf * k_eff + (1.0 - lf) * k_eff;
    kf = kf + (lf * 0.0 + (1.0 - lf) * 0.0);
    const double area = d.area[f];
    const double DT = P.nonorth_corr > 0.0 ? kf * (area * area) / d.dsf[f] : kf * area / d.dn[f];
    const double off = own ? DT + fmax(-FT, 0.0) : DT + fmax(FT, 0.0);
    ap = own ? ap + fmax(FT, 0.0) + DT : ap + fmax(-FT, 0.0) + DT;
    const int slot = d.cf_slot[k];
    A[slot] = (d.cf_first[k] ? 0.0 : A[slot]) - off;
    if (P.conv_blend > 0.0) {
      const int cu = (FT > 0.0) ? a : b;
      const double dc = P.conv_blend * FT *
                        (d.psiT[cu] * dot3(d.gt[cu], d.gt[N + cu], d.gt[2 * N + cu], d.xf[f] - d.xc[cu],
                                           d.xf[F + f] - d.xc[N + cu], d.xf[2 * F + f] - d.xc[2 * N + cu]));
      rhs = own ? rhs - dc : rhs + dc;
    }
    if (P.nonorth_corr > 0.0) {
      const double l1 = 1.0 - lf;
      const double gf0 = lf * d.gt[a] + l1 * d.gt[b];
      const double gf1 = lf * d.gt[N + a] + l1 * d.gt[N + b];
      const double gf2 = lf * d.gt[2 * N + a] + l1 * d.gt[2 * N + b];
      const double noc = P.nonorth_corr * kf * dot3(gf0, gf1, gf2, d.tv[f], d.tv[F + f], d.tv[2 * F + f]);
      rhs = own ? rhs + noc : rhs - noc;
    }
  }
  const double tc = d.T[c];
  for (int k = kb; k < ke; ++k) {
    const int f = d.cf[k];
    if (d.c1[f] >= 0) continue;
    const DevGroup& g = d.groups[d.fgrp[f]];
    double T_face, q_face;
    bool neu;
    bc_face_T(g, thermal_iface(d), f, d.xf[f], d.xf[F + f], d.xf[2 * F + f], tc, T_face, q_face, neu);
    double kf = 1.0 * P.k_cond + (1.0 - 1.0) * 0.0;
    kf = kf + 0.0;
    const double DT = kf * d.area[f] / d.dn[f];
    const double FT = P.cp * d.flux[f];
    if (!neu) {
      ap = ap + DT + fmax(FT, 0.0);
      rhs = rhs + DT * T_face - fmin(FT, 0.0) * T_face;
    } else {
      if (fabs(q_face) > 0.0) rhs = rhs + q_face * d.area[f];
      if (g.btype == MGPU_BC_POUTLET || g.btype == MGPU_BC_OUTFLOW) ap = ap + fmax(FT, 0.0);
    }
  }
  const double vol = d.vol[c];
  const int ts = d.st->ts_order;
  if (ts == 1) {
    const double at = (1.0 * P.rho * P.cp + (1.0 - 1.0) * 0.0 * 0.0) * vol / P.dt;
    ap = ap + at;
    rhs = rhs + at * d.T_old[c];
  } else if (ts == 2) {
    const double at = (1.0 * P.rho * P.cp + (1.0 - 1.0) * 0.0 * 0.0) * vol / (2.0 * P.dt);
    ap = ap + 3.0 * at;
    rhs = rhs + at * (4.0 * d.T_old[c] - d.T_old_old[c]);
  }
  if (ts > 0 && !P.pimple) {
    A[d.diag[c]] = ap;
  } else {
    A[d.diag[c]] = ap / P.alpha_u;
    rhs = rhs + (1.0 - P.alpha_u) / P.alpha_u * ap * tc;
  }
  d.rhs[c] = rhs;
  d.ap[c] = ap;
}
__global__ void __launch_bounds__(256) k_temperature(DeviceCase d, AsmParams P) {
  b_temperature(d, P, blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------- batched launches -----------------------------------------
// One launch runs a kernel over many cases. Block b belongs to case
// blk_case[range][b] and acts as block b - blk0[range] of that case's own
// launch of the same body, so every case computes exactly what its
// single-case launch computes. The case's descriptor is staged in shared
// memory once per block.

__device__ __forceinline__ const BatchCase& stage_case(unsigned char* raw, const BatchCase* src) {
  constexpr int W = (int)(sizeof(BatchCase) / 8);
  const long long* s = reinterpret_cast<const long long*>(src);
  long long* t = reinterpret_cast<long long*>(raw);
  for (int k = threadIdx.x; k < W; k += blockDim.x) t[k] = s[k];
  __syncthreads();
  return *reinterpret_cast<const BatchCase*>(raw);
}

#define MGPU_BATCHED(NAME, RANGE, ...)                                                 \
  __global__ void __launch_bounds__(256) kb_##NAME(AsmBatch B, int arg) {              \
    __shared__ __align__(16) unsigned char raw[sizeof(BatchCase)];                     \
    const BatchCase& sc = stage_case(raw, B.cases + B.blk_case[RANGE][blockIdx.x]);    \
    const DeviceCase& d = sc.d;                                                        \
    const AsmParams& P = sc.P;                                                         \
    const long i = (long)(blockIdx.x - sc.blk0[RANGE]) * blockDim.x + threadIdx.x;     \
    (void)arg;                                                                         \
    (void)i;                                                                           \
    (void)P;                                                                           \
    __VA_ARGS__;                                                                       \
  }

MGPU_BATCHED(fill_apc, RANGE_N, if (i < d.N) d.apc[i] = 1.0)
MGPU_BATCHED(gradients, RANGE_N, b_gradients<1>(d, P, (int)i))
MGPU_BATCHED(rhiechow_piso, RANGE_F, if (sc.transient) b_rhiechow(d, P, (int)i))
MGPU_BATCHED(begin_iter, RANGE_3N, b_begin_iter(d, sc.transient, sc.time_scheme, P.inlet_ramp, i))
MGPU_BATCHED(limiter, RANGE_N, if (P.conv_blend > 0.0) b_limiter(d, P, arg, (int)i))
MGPU_BATCHED(momentum, RANGE_N, b_momentum(d, P, arg, (int)i))
MGPU_BATCHED(mom_interior, RANGE_N, b_mom_interior<2>(d, P, (int)i))
MGPU_BATCHED(mom_finish, RANGE_N, b_mom_finish(d, P, arg, (int)i))
MGPU_BATCHED(apc, RANGE_N, b_apc(d, sc.transient ? 1.0 : P.alpha_u, (int)i))
MGPU_BATCHED(rhiechow, RANGE_F, b_rhiechow(d, P, (int)i))
MGPU_BATCHED(outflow, RANGE_ONE, if (sc.has_outflow) b_outflow(d))
MGPU_BATCHED(ppe, RANGE_N, if (arg < sc.ncorr) b_ppe<2>(d, P, (int)i))
MGPU_BATCHED(correct_cells, RANGE_N, if (arg < sc.ncorr) b_correct_cells<2>(d, P, (int)i))
MGPU_BATCHED(correct_flux, RANGE_F, if (arg < sc.ncorr) b_correct_flux(d, (int)i))
MGPU_BATCHED(diag, RANGE_N, b_diag(d, sc.transient, (int)i))
MGPU_BATCHED(diag_finalize, RANGE_ONE, if (threadIdx.x == 0) b_diag_finalize(d, P, sc.transient))

#undef MGPU_BATCHED

}  // namespace

// ---------------- launchers -------------------------------------------------

#define GRID(n) ceil_div((n), 256), 256, 0, s
// a cell-gather kernel KERNEL<k> for chunk size k: the gather_faces key if
// set, else the kernel's own measured best DEF (B200, 524k channel: 1 for the
// gradients, 2 for the momentum interior, PPE and cell correction)
#define MGPU_GATHER_LAUNCH(KERNEL, DEF, ...)                    \
  do {                                                          \
    const int k_ = g_gather_faces > 0 ? g_gather_faces : (DEF); \
    if (k_ >= 6)                                                \
      KERNEL<6 __VA_ARGS__><<<GRID(d.N)>>>(d, P);               \
    else if (k_ >= 3)                                           \
      KERNEL<3 __VA_ARGS__><<<GRID(d.N)>>>(d, P);               \
    else if (k_ == 2)                                           \
      KERNEL<2 __VA_ARGS__><<<GRID(d.N)>>>(d, P);               \
    else                                                        \
      KERNEL<1 __VA_ARGS__><<<GRID(d.N)>>>(d, P);               \
  } while (0)

int geometry_setup(DeviceCase& d, const double* x, const int* fptr, const int* fnodes, double* pcen,
                   const AsmParams& P, cudaStream_t s) {
  k_face_props<<<GRID(d.F)>>>(d.F, x, fptr, fnodes, d.xf, d.sf, d.area);
  MGPU_LAUNCH_CHECK("k_face_props");
  k_prov_centers<<<GRID(d.N)>>>(d.N, x, fptr, fnodes, d.cf_ptr, d.cf, pcen);
  MGPU_LAUNCH_CHECK("k_prov_centers");
  k_orient<<<GRID(d.F)>>>(d.F, d.N, d.c0, d.xf, pcen, d.sf);
  MGPU_LAUNCH_CHECK("k_orient");
  k_cell_volumes<<<GRID(d.N)>>>(d.N, d.F, d.c0, d.cf_ptr, d.cf, d.xf, d.sf, pcen, d.vol, d.xc);
  MGPU_LAUNCH_CHECK("k_cell_volumes");
  k_face_consts<<<GRID(d.F)>>>(d, P);
  MGPU_LAUNCH_CHECK("k_face_consts");
  return 0;
}

int launch_gradients(const DeviceCase& d, const AsmParams& P, cudaStream_t s) {
  MGPU_GATHER_LAUNCH(k_gradients, 1);
  MGPU_LAUNCH_CHECK("k_gradients");
  if (d.energy) {
    k_tgrad<<<GRID(d.N)>>>(d);
    MGPU_LAUNCH_CHECK("k_tgrad");
  }
  return 0;
}

int launch_temperature(const DeviceCase& d, const AsmParams& P, cudaStream_t s) {
  if (P.conv_blend > 0.0) {
    k_tlimiter<<<GRID(d.N)>>>(d);
    MGPU_LAUNCH_CHECK("k_tlimiter");
  }
  k_temperature<<<GRID(d.N)>>>(d, P);
  MGPU_LAUNCH_CHECK("k_temperature");
  return 0;
}
int launch_limiter(const DeviceCase& d, const AsmParams& P, int comp, cudaStream_t s) {
  k_limiter<<<GRID(d.N)>>>(d, P, comp);
  MGPU_LAUNCH_CHECK("k_limiter");
  return 0;
}
int launch_momentum(const DeviceCase& d, const AsmParams& P, int comp, cudaStream_t s) {
  k_momentum<<<GRID(d.N)>>>(d, P, comp);
  MGPU_LAUNCH_CHECK("k_momentum");
  return 0;
}
int launch_mom_interior(const DeviceCase& d, const AsmParams& P, cudaStream_t s) {
  if (P.nonorth_corr > 0.0)
    MGPU_GATHER_LAUNCH(k_mom_interior, 2, , true);
  else
    MGPU_GATHER_LAUNCH(k_mom_interior, 2, , false);
  MGPU_LAUNCH_CHECK("k_mom_interior");
  return 0;
}
int launch_mom_finish(const DeviceCase& d, const AsmParams& P, int comp, cudaStream_t s) {
  k_mom_finish<<<GRID(d.N)>>>(d, P, comp);
  MGPU_LAUNCH_CHECK("k_mom_finish");
  return 0;
}
int launch_apc(const DeviceCase& d, double div, cudaStream_t s) {
  k_apc<<<GRID(d.N)>>>(d, div);
  MGPU_LAUNCH_CHECK("k_apc");
  return 0;
}
int launch_fill(double* a, long n, double v, cudaStream_t s) {
  k_fill<<<GRID(n)>>>(a, n, v);
  MGPU_LAUNCH_CHECK("k_fill");
  return 0;
}
int launch_rhiechow(const DeviceCase& d, const AsmParams& P, cudaStream_t s) {
  k_rhiechow<<<GRID(d.F)>>>(d, P);
  MGPU_LAUNCH_CHECK("k_rhiechow");
  return 0;
}
int launch_outflow(const DeviceCase& d, cudaStream_t s) {
  k_outflow<<<1, 256, 0, s>>>(d);
  MGPU_LAUNCH_CHECK("k_outflow");
  return 0;
}
int launch_ppe(const DeviceCase& d, const AsmParams& P, cudaStream_t s) {
  MGPU_GATHER_LAUNCH(k_ppe, 2);
  MGPU_LAUNCH_CHECK("k_ppe");
  return 0;
}
int launch_correct(const DeviceCase& d, const AsmParams& P, cudaStream_t s) {
  MGPU_GATHER_LAUNCH(k_correct_cells, 2);
  MGPU_LAUNCH_CHECK("k_correct_cells");
  k_correct_flux<<<GRID(d.F)>>>(d);
  MGPU_LAUNCH_CHECK("k_correct_flux");
  return 0;
}
int launch_diag(const DeviceCase& d, const AsmParams& P, int transient, cudaStream_t s) {
  k_diag<<<GRID(d.N)>>>(d, transient);
  MGPU_LAUNCH_CHECK("k_diag");
  k_diag_finalize<<<1, 1, 0, s>>>(d, P, transient);
  MGPU_LAUNCH_CHECK("k_diag_finalize");
  return 0;
}

int launch_outer_accum(const DeviceCase& d, cudaStream_t s) {
  k_outer_accum<<<1, 1, 0, s>>>(d);
  MGPU_LAUNCH_CHECK("k_outer_accum");
  return 0;
}
int launch_batch_asm(int op, int arg, const AsmBatch& b, cudaStream_t s) {
  struct OpInfo {
    void (*fn)(AsmBatch, int);
    int range;
    const char* name;
  };
  static const OpInfo ops[BOP_COUNT] = {
      {kb_fill_apc, RANGE_N, "kb_fill_apc"},
      {kb_gradients, RANGE_N, "kb_gradients"},
      {kb_rhiechow_piso, RANGE_F, "kb_rhiechow_piso"},
      {kb_begin_iter, RANGE_3N, "kb_begin_iter"},
      {kb_limiter, RANGE_N, "kb_limiter"},
      {kb_momentum, RANGE_N, "kb_momentum"},
      {kb_mom_interior, RANGE_N, "kb_mom_interior"},
      {kb_mom_finish, RANGE_N, "kb_mom_finish"},
      {kb_apc, RANGE_N, "kb_apc"},
      {kb_rhiechow, RANGE_F, "kb_rhiechow"},
      {kb_outflow, RANGE_ONE, "kb_outflow"},
      {kb_ppe, RANGE_N, "kb_ppe"},
      {kb_correct_cells, RANGE_N, "kb_correct_cells"},
      {kb_correct_flux, RANGE_F, "kb_correct_flux"},
      {kb_diag, RANGE_N, "kb_diag"},
      {kb_diag_finalize, RANGE_ONE, "kb_diag_finalize"},
  };
  if (op < 0 || op >= BOP_COUNT) {
    set_error("launch_batch_asm: unknown op");
    return MGPU_E_ARG;
  }
  const OpInfo& o = ops[op];
  if (b.nblk[o.range] <= 0) return 0;
  o.fn<<<b.nblk[o.range], 256, 0, s>>>(b, arg);
  MGPU_LAUNCH_CHECK(o.name);
  return 0;
}

int launch_begin_iter(const DeviceCase& d, int transient, int time_scheme, int inlet_ramp, cudaStream_t s) {
  k_begin_iter<<<GRID(3l * d.N)>>>(d, transient, time_scheme, inlet_ramp);
  MGPU_LAUNCH_CHECK("k_begin_iter");
  return 0;
}

}  // namespace mgpu
