// krylov_mixed.cu -- mixed-precision form of the Krylov solves.
//
// FP64 iterative refinement around an FP32 inner Krylov method:
//   r = b - A x                      (FP64 SpMV, FP64 accumulation)
//   solve A d = r / |r| to tau        (FP32 matrix and vectors, FP32 SpMV
//                                      accumulation, Jacobi preconditioner in
//                                      FP32; every dot product and norm in FP64)
//   x += |r| d                        (FP64)
// until |b - A x| / |b| <= tol (the true residual, recomputed in FP64). The
// matrix is rounded to FP32 inside the same launch. One cooperative launch
// per solve, as in the FP64 form; `it` counts inner iterations.
//
// This form does not reproduce the reference's iteration counts (different
// preconditioner, different precision); it converges the same systems to the
// same tolerance on the true residual.

#include <algorithm>

#include "persist.cuh"

namespace mgpu {
namespace {

template <bool L1>
__device__ __forceinline__ float row_spmv32(const int* __restrict__ rp, const int* __restrict__ col,
                                            const float* __restrict__ val, const float* x, int i) {
  float y = 0.0f;
  const int e = rp[i + 1];
  for (int k = rp[i]; k < e; ++k) y = fmaf(val[k], ldv<L1>(&x[col[k]]), y);
  return y;
}

// q = A32 x for the rows i0, i0 + stride, ... (up to R rows per thread),
// issuing every row's loads before any accumulation, so R rows' memory
// latencies overlap. FP32 accumulation in CSR order.
template <bool L1, int R, int MAXNZ>
__device__ __forceinline__ void spmv32_rows(const int* __restrict__ rp, const int* __restrict__ col,
                                            const float* __restrict__ val, const float* x, int i0, int stride,
                                            int n, float (&y)[R]) {
  int b[R], e[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = i0 + r * stride;
    b[r] = i < n ? rp[i] : 0;
    e[r] = i < n ? rp[i + 1] : 0;
  }
  float v[R][MAXNZ];
  int c[R][MAXNZ];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int t = 0; t < MAXNZ; ++t)
      if (b[r] + t < e[r]) {
        c[r][t] = col[b[r] + t];
        v[r][t] = val[b[r] + t];
      }
  float xv[R][MAXNZ];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int t = 0; t < MAXNZ; ++t)
      if (b[r] + t < e[r]) xv[r][t] = ldv<L1>(&x[c[r][t]]);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    float acc = 0.0f;
#pragma unroll
    for (int t = 0; t < MAXNZ; ++t)
      if (b[r] + t < e[r]) acc = fmaf(v[r][t], xv[r][t], acc);
    for (int k = b[r] + MAXNZ; k < e[r]; ++k) acc = fmaf(val[k], ldv<L1>(&x[col[k]]), acc);
    y[r] = acc;
  }
}

// The same product from the column-major ELL copy: entry t of row i sits at
// t*n + i, so a warp's loads of one t are contiguous and no row pointer is
// read. Padding entries have value 0 and the row's own column.
template <bool L1, int R>
__device__ __forceinline__ void spmv32_ell(const MixedArgs& m, const float* x, int i0, int stride, int n,
                                           float (&y)[R]) {
  constexpr int WMAX = 8;
  const int W = m.ell_w;
  float v[R][WMAX];
  int c[R][WMAX];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = i0 + r * stride;
#pragma unroll
    for (int t = 0; t < WMAX; ++t)
      if (t < W && i < n) {
        c[r][t] = m.ell_col[(long)t * n + i];
        v[r][t] = m.ell_val[(long)t * n + i];
      }
  }
  float xv[R][WMAX];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int t = 0; t < WMAX; ++t)
      if (t < W && i0 + r * stride < n) xv[r][t] = ldv<L1>(&x[c[r][t]]);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    float acc = 0.0f;
#pragma unroll
    for (int t = 0; t < WMAX; ++t)
      if (t < W && i0 + r * stride < n) acc = fmaf(v[r][t], xv[r][t], acc);
    y[r] = acc;
  }
}

template <bool L1, bool ELL, int R>
__device__ __forceinline__ void spmv32_any(const KrylovArgs& a, const MixedArgs& m, const float* x, int i0,
                                           int stride, int n, float (&y)[R]) {
  if constexpr (ELL)
    spmv32_ell<L1, R>(m, x, i0, stride, n, y);
  else
    spmv32_rows<L1, R, 8>(a.row_ptr, a.col, m.a32, x, i0, stride, n, y);
}

template <bool L1>
__device__ __forceinline__ double row_spmv64(const KrylovArgs& a, const double* x, int i) {
  double y = 0.0;
  const int e = a.row_ptr[i + 1];
  for (int k = a.row_ptr[i]; k < e; ++k) y = fma(a.aval[k], ldv<L1>(&x[a.col[k]]), y);
  return y;
}

__device__ void write_result_m(const KrylovArgs& a, int it, double res, int ierr) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    MgpuIterRec* rec = a.recs + a.st->cur_it;
    if (a.slot >= 0 && a.slot < MGPU_MAXSOLVE) {
      rec->lin_it[a.slot] = it;
      rec->lin_res[a.slot] = res;
      rec->lin_ierr[a.slot] = ierr;
      if (rec->nsolve < a.slot + 1) rec->nsolve = a.slot + 1;
    }
    if (ierr == 2 && a.ier_breakdown != 0) {
      a.st->ier = a.ier_breakdown;
      a.st->abort = 1;
    }
  }
}

// Shared prologue: FP32 copy of A, FP32 inverse diagonal, b.b; returns false
// when the kernel must leave (barrier timeout).
template <bool L1>
__device__ bool prologue(const KrylovArgs& a, const MixedArgs& m, double& bnrm, bool& diag_bad) {
  const int n = a.n, nnz = a.row_ptr[n];
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstr = gridDim.x * blockDim.x;
  for (int k = gtid; k < nnz; k += gstr) m.a32[k] = (float)a.aval[k];
  double v[2] = {0.0, 0.0};
  for (int i = gtid; i < n; i += gstr) {
    if (m.ell_col) {
      const int rb = a.row_ptr[i], len = a.row_ptr[i + 1] - rb;
      for (int t = 0; t < m.ell_w; ++t) m.ell_val[(long)t * n + i] = t < len ? (float)a.aval[rb + t] : 0.0f;
    }
    if (a.zero_x) a.x[i] = 0.0;
    const double dg = a.aval[a.diag[i]];
    if (fabs(dg) < DTINY) v[1] = v[1] + 1.0;
    m.dinv[i] = (float)(1.0 / dg);
    v[0] = fma(a.b[i], a.b[i], v[0]);
  }
  if (!grid_sum<2, L1>(v, a.partials, a.bar, a.st)) return false;
  bnrm = sqrt(v[0]);
  diag_bad = v[1] != 0.0;
  return true;
}

// r = b - A x in FP64; returns |r| through rnorm
template <bool L1>
__device__ bool true_residual(const KrylovArgs& a, double& rnorm) {
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstr = gridDim.x * blockDim.x;
  double v[1] = {0.0};
  for (int i = gtid; i < a.n; i += gstr) {
    const double ri = a.b[i] - row_spmv64<L1>(a, a.x, i);
    a.r[i] = ri;
    v[0] = fma(ri, ri, v[0]);
  }
  if (!grid_sum<1, L1>(v, a.partials, a.bar, a.st)) return false;
  rnorm = sqrt(v[0]);
  return true;
}

// x += scale * d, then a barrier (neighbours' x are read next)
template <bool L1>
__device__ bool update_x(const KrylovArgs& a, const float* d, double scale) {
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstr = gridDim.x * blockDim.x;
  for (int i = gtid; i < a.n; i += gstr) a.x[i] = fma(scale, (double)d[i], a.x[i]);
  return grid_sync(a.bar, a.st);
}

// Chebyshev-Jacobi preconditioner z = p(D^-1 A) D^-1 rr of degree k on
// [lmax/ratio, lmax]: k-1 SpMV passes, one barrier each, no reductions.
// On entry z0 = d = D^-1 rr / theta (written by the caller's pass, followed by
// a barrier). The result lands in zout (z0 or z1, ping-pong); the last pass
// also accumulates rr.z and rr.rr, reduced before returning.
template <bool L1, bool ELL>
__device__ bool cheb_apply(const KrylovArgs& a, const MixedArgs& m, const float* rr, float* dch, float* z0,
                           float* z1, double lmax, float*& zout, double (&red)[2]) {
  const int n = a.n;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstr = gridDim.x * blockDim.x;
  const double lmin = lmax / m.cheb_ratio;
  const double th = 0.5 * (lmax + lmin), de = 0.5 * (lmax - lmin), sg = th / de;
  double rho0 = 1.0 / sg;
  float* zc = z0;
  float* zn = z1;
  red[0] = red[1] = 0.0;
  for (int j = 1; j < m.cheb_k; ++j) {
    const double rho1 = 1.0 / (2.0 * sg - rho0);
    const float c1 = (float)(rho1 * rho0), c2 = (float)(2.0 * rho1 / de);
    const bool last = (j == m.cheb_k - 1);
    constexpr int R = ELL ? 1 : 2;
    for (int i0 = gtid; i0 < n; i0 += R * gstr) {
      float az[R];
      spmv32_any<L1, ELL, R>(a, m, zc, i0, gstr, n, az);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = i0 + r * gstr;
        if (i < n) {
          const float res = m.dinv[i] * (rr[i] - az[r]);
          const float dn = fmaf(c1, dch[i], c2 * res);
          dch[i] = dn;
          const float zi = zc[i] + dn;
          zn[i] = zi;
          if (last) {
            red[0] = fma((double)rr[i], (double)zi, red[0]);
            red[1] = fma((double)rr[i], (double)rr[i], red[1]);
          }
        }
      }
    }
    if (last) {
      if (!grid_sum<2, L1>(red, a.partials, a.bar, a.st)) return false;
    } else if (!grid_sync(a.bar, a.st)) {
      return false;
    }
    float* t = zc;
    zc = zn;
    zn = t;
    rho0 = rho1;
  }
  zout = zc;
  return true;
}

template <bool L1, bool ELL>
__global__ void __launch_bounds__(L1 ? 512 : 256, L1 ? 1 : 2) k_pcg_mixed(KrylovArgs a, MixedArgs m) {
  if (a.st->abort) return;
  const int n = a.n;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstr = gridDim.x * blockDim.x;
  float *rr = m.w32, *zA = m.w32 + n, *p = m.w32 + 2l * n, *q = m.w32 + 3l * n, *d = m.w32 + 4l * n;
  float *dch = m.w32 + 5l * n, *zB = m.w32 + 6l * n;
  const bool cheb = m.cheb_k > 1;
  double bnrm;
  bool diag_bad;
  if (!prologue<L1>(a, m, bnrm, diag_bad)) return;
  if (bnrm == 0.0) {
    for (int i = gtid; i < n; i += gstr) a.x[i] = 0.0;
    write_result_m(a, 0, 0.0, 0);
    return;
  }
  if (diag_bad) {
    write_result_m(a, 0, 0.0, 2);
    return;
  }
  // Chebyshev interval: Gershgorin bound of D^-1 A (row sum of |a_ij| / a_ii)
  double lmax = 2.0, th = 1.0;
  if (cheb) {
    double g = 0.0;
    for (int i = gtid; i < n; i += gstr) {
      double s = 0.0;
      for (int k = a.row_ptr[i]; k < a.row_ptr[i + 1]; ++k) s += fabs(a.aval[k]);
      g = fmax(g, s / fabs(a.aval[a.diag[i]]));
    }
    if (!grid_max<L1>(g, a.partials, a.bar, a.st)) return;
    lmax = g;
    th = 0.5 * (lmax + lmax / m.cheb_ratio);
  }
  const float inv_th = (float)(1.0 / th);
  double rnorm;
  if (!true_residual<L1>(a, rnorm)) return;
  double res = rnorm / bnrm;
  if (res <= a.tol) {
    write_result_m(a, 0, res, 0);
    return;
  }
  int total = 0, ierr = 0;
  float* z = zA;
  while (true) {
    // restart on the scaled FP64 residual
    const double inv = 1.0 / rnorm;
    double v2[2] = {0.0, 0.0};
    for (int i = gtid; i < n; i += gstr) {
      const float ri = (float)(ldv<L1>(&a.r[i]) * inv);
      rr[i] = ri;
      d[i] = 0.0f;
      if (cheb) {
        const float di = m.dinv[i] * ri * inv_th;
        dch[i] = di;
        zA[i] = di;
      } else {
        const float zi = m.dinv[i] * ri;
        zA[i] = zi;
        v2[0] = fma((double)ri, (double)zi, v2[0]);
        v2[1] = fma((double)ri, (double)ri, v2[1]);
      }
    }
    if (cheb) {
      if (!grid_sync(a.bar, a.st)) return;
      if (!cheb_apply<L1, ELL>(a, m, rr, dch, zA, zB, lmax, z, v2)) return;
    } else {
      z = zA;
      if (!grid_sum<2, L1>(v2, a.partials, a.bar, a.st)) return;
    }
    double rz = v2[0];
    const double target = m.tau * m.tau * v2[1];
    // p := z and q := A p on the first inner iteration; afterwards
    // p := z + beta p and q := A z + beta q in the same pass
    float beta = 0.0f;
    bool first = true;
    while (true) {
      ++total;
      double pq[1] = {0.0};
      constexpr int R = ELL ? 1 : 2;
      for (int i0 = gtid; i0 < n; i0 += R * gstr) {
        float az[R];
        spmv32_any<L1, ELL, R>(a, m, z, i0, gstr, n, az);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = i0 + r * gstr;
          if (i < n) {
            const float pi = first ? z[i] : fmaf(beta, p[i], z[i]);
            const float qi = first ? az[r] : fmaf(beta, q[i], az[r]);
            p[i] = pi;
            q[i] = qi;
            pq[0] = fma((double)pi, (double)qi, pq[0]);
          }
        }
      }
      first = false;
      if (!grid_sum<1, L1>(pq, a.partials, a.bar, a.st)) return;
      if (fabs(pq[0]) < DTINY) {
        ierr = 2;
        break;
      }
      const double alpha = rz / pq[0];
      const float af = (float)alpha;
      double u2[2] = {0.0, 0.0};
      for (int i = gtid; i < n; i += gstr) {
        d[i] = fmaf(af, p[i], d[i]);
        const float ri = fmaf(-af, q[i], rr[i]);
        rr[i] = ri;
        if (cheb) {
          const float di = m.dinv[i] * ri * inv_th;
          dch[i] = di;
          zA[i] = di;
        } else {
          const float zi = m.dinv[i] * ri;
          zA[i] = zi;
          u2[0] = fma((double)ri, (double)ri, u2[0]);
          u2[1] = fma((double)ri, (double)zi, u2[1]);
        }
      }
      if (cheb) {
        if (!grid_sync(a.bar, a.st)) return;
        double red[2];
        if (!cheb_apply<L1, ELL>(a, m, rr, dch, zA, zB, lmax, z, red)) return;
        u2[0] = red[1];
        u2[1] = red[0];
      } else {
        z = zA;
        if (!grid_sum<2, L1>(u2, a.partials, a.bar, a.st)) return;
      }
      if (u2[0] <= target || total >= a.maxit) break;
      if (fabs(rz) < DTINY) {
        ierr = 2;
        break;
      }
      beta = (float)(u2[1] / rz);
      rz = u2[1];
    }
    if (ierr == 2) break;
    if (!update_x<L1>(a, d, rnorm)) return;
    if (!true_residual<L1>(a, rnorm)) return;
    res = rnorm / bnrm;
    if (res <= a.tol) {
      write_result_m(a, total, res, 0);
      return;
    }
    if (total >= a.maxit) {
      ierr = 1;
      break;
    }
  }
  write_result_m(a, total, res, ierr);
}

template <bool L1>
__global__ void __launch_bounds__(L1 ? 512 : 256) k_bicgstab_mixed(KrylovArgs a, MixedArgs m) {
  if (a.st->abort) return;
  const int n = a.n;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstr = gridDim.x * blockDim.x;
  float* W = m.w32;
  float *r = W, *r0 = W + n, *p = W + 2l * n, *v = W + 3l * n, *s = W + 4l * n, *t = W + 5l * n,
        *ph = W + 6l * n, *sh = W + 7l * n, *d = W + 8l * n;
  double bnrm;
  bool diag_bad;
  if (!prologue<L1>(a, m, bnrm, diag_bad)) return;
  if (bnrm == 0.0) {
    for (int i = gtid; i < n; i += gstr) a.x[i] = 0.0;
    write_result_m(a, 0, 0.0, 0);
    return;
  }
  if (diag_bad) {
    write_result_m(a, 0, 0.0, 12);
    return;
  }
  double rnorm;
  if (!true_residual<L1>(a, rnorm)) return;
  double res = rnorm / bnrm;
  if (res <= a.tol) {
    write_result_m(a, 0, res, 0);
    return;
  }
  int total = 0, ierr = 0;
  while (true) {
    const double inv = 1.0 / rnorm;
    double w1[1] = {0.0};
    for (int i = gtid; i < n; i += gstr) {
      const float ri = (float)(ldv<L1>(&a.r[i]) * inv);
      r[i] = ri;
      r0[i] = ri;
      p[i] = 0.0f;
      v[i] = 0.0f;
      d[i] = 0.0f;
      w1[0] = fma((double)ri, (double)ri, w1[0]);
    }
    if (!grid_sum<1, L1>(w1, a.partials, a.bar, a.st)) return;
    const double target = m.tau * m.tau * w1[0];
    double rho_next = w1[0], rho_old = 1.0, alpha = 1.0, omega = 1.0;
    while (true) {
      ++total;
      const double rho = rho_next;
      if (fabs(rho) < DTINY) {
        ierr = 2;
        break;
      }
      const float beta = (float)((rho / rho_old) * (alpha / omega));
      const float om = (float)omega;
      for (int i = gtid; i < n; i += gstr) {
        const float pi = fmaf(beta, fmaf(-om, v[i], p[i]), r[i]);
        p[i] = pi;
        ph[i] = m.dinv[i] * pi;
      }
      if (!grid_sync(a.bar, a.st)) return;
      double d1[1] = {0.0};
      for (int i = gtid; i < n; i += gstr) {
        const float vi = row_spmv32<L1>(a.row_ptr, a.col, m.a32, ph, i);
        v[i] = vi;
        d1[0] = fma((double)r0[i], (double)vi, d1[0]);
      }
      if (!grid_sum<1, L1>(d1, a.partials, a.bar, a.st)) return;
      alpha = rho / d1[0];
      const float af = (float)alpha;
      double d2[1] = {0.0};
      for (int i = gtid; i < n; i += gstr) {
        const float si = fmaf(-af, v[i], r[i]);
        s[i] = si;
        sh[i] = m.dinv[i] * si;
        d2[0] = fma((double)si, (double)si, d2[0]);
      }
      if (!grid_sum<1, L1>(d2, a.partials, a.bar, a.st)) return;
      if (d2[0] <= target || total >= a.maxit) {
        for (int i = gtid; i < n; i += gstr) d[i] = fmaf(af, ph[i], d[i]);
        break;
      }
      double d3[2] = {0.0, 0.0};
      for (int i = gtid; i < n; i += gstr) {
        const float ti = row_spmv32<L1>(a.row_ptr, a.col, m.a32, sh, i);
        t[i] = ti;
        d3[0] = fma((double)ti, (double)ti, d3[0]);
        d3[1] = fma((double)ti, (double)s[i], d3[1]);
      }
      if (!grid_sum<2, L1>(d3, a.partials, a.bar, a.st)) return;
      if (d3[0] < DTINY) {
        ierr = 2;
        break;
      }
      omega = d3[1] / d3[0];
      if (fabs(omega) < DTINY) {
        ierr = 2;
        break;
      }
      const float omf = (float)omega;
      double d4[2] = {0.0, 0.0};
      for (int i = gtid; i < n; i += gstr) {
        d[i] = fmaf(omf, sh[i], fmaf(af, ph[i], d[i]));
        const float ri = fmaf(-omf, t[i], s[i]);
        r[i] = ri;
        d4[0] = fma((double)ri, (double)ri, d4[0]);
        d4[1] = fma((double)ri, (double)r0[i], d4[1]);
      }
      if (!grid_sum<2, L1>(d4, a.partials, a.bar, a.st)) return;
      if (d4[0] <= target || total >= a.maxit) break;
      rho_next = d4[1];
      rho_old = rho;
    }
    if (ierr == 2) break;
    if (!update_x<L1>(a, d, rnorm)) return;
    if (!true_residual<L1>(a, rnorm)) return;
    res = rnorm / bnrm;
    if (res <= a.tol) {
      write_result_m(a, total, res, 0);
      return;
    }
    if (total >= a.maxit) {
      ierr = 1;
      break;
    }
  }
  write_result_m(a, total, res, ierr);
}

int launch_mixed(const void* fn1, const void* fnN, const KrylovArgs& a, const MixedArgs& m, cudaStream_t s) {
  int block = 0;
  int grid = krylov_grid(a.n, block, 0);
  if (grid > 1) {  // this kernel's own co-residency; about 2 rows per thread
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fnN, block, 0);
    if (per < 1) per = 1;
    long want = ((long)a.n + 2l * block - 1) / (2l * block);
    grid = (int)std::min<long>(std::max<long>(want, 2), (long)sms * per);
  }
  KrylovArgs aa = a;
  MixedArgs mm = m;
  void* args[] = {&aa, &mm};
  cudaError_t e = cudaMemsetAsync(a.bar, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return cuda_fail(e, "barrier reset", __FILE__, __LINE__);
  e = cudaLaunchCooperativeKernel(grid == 1 ? fn1 : fnN, dim3(grid), dim3(block), args, 0, s);
  if (e != cudaSuccess) return cuda_fail(e, "cooperative launch (mixed)", __FILE__, __LINE__);
  return 0;
}

}  // namespace

int launch_pcg_mixed(const KrylovArgs& a, const MixedArgs& m, cudaStream_t s) {
  if (m.ell_col)
    return launch_mixed((const void*)k_pcg_mixed<true, true>, (const void*)k_pcg_mixed<false, true>, a, m, s);
  return launch_mixed((const void*)k_pcg_mixed<true, false>, (const void*)k_pcg_mixed<false, false>, a, m, s);
}

int launch_bicgstab_mixed(const KrylovArgs& a, const MixedArgs& m, cudaStream_t s) {
  return launch_mixed((const void*)k_bicgstab_mixed<true>, (const void*)k_bicgstab_mixed<false>, a, m, s);
}

}  // namespace mgpu
