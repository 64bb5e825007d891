// krylov.cu -- persistent Krylov solves of the FP64 parity form.
//
// One cooperative kernel per linear solve (PCG or BiCGStab): every phase of
// the reference's iteration runs as a grid-stride pass, dot products and norms
// are two-level deterministic reductions (warp butterfly + fixed-order sum of
// per-block partials), and the phases are separated by a bounded grid barrier,
// so the Krylov scalars never leave the GPU and the solve costs one launch.
// ILU(0)/IC(0) factorisation and triangular sweeps are level-scheduled: rows
// of one level are independent, and each row is computed by one thread in the
// reference's sequential order, so factor values and sweep results are
// bit-identical to mod_uns_linsolver.f90.
//
// Reference: src/unstructured/mod_uns_linsolver.f90 (csr_matvec :40-52,
// ilu0_factor :79-115, ilu0_apply :120-142, bicgstab_ilu0 :148-224, cg_jacobi
// :230-291, ic0_factor :328-365, ic0_apply :371-399, cg_ic0 :405-461) and
// mod_uns_linsolver_mpi.f90:155-363 at one rank.

#include <type_traits>

#include "persist.cuh"

namespace mgpu {

namespace {


// y_i = A_i . x in csr_matvec order (x may have been written by other blocks).
template <bool L1>
__device__ __forceinline__ double row_spmv(const int* __restrict__ rp, const int* __restrict__ col,
                                           const double* __restrict__ val, const double* x, int i) {
  double y = 0.0;
  const int e = rp[i + 1];
  for (int k = rp[i]; k < e; ++k) y = y + val[k] * ldv(&x[col[k]]);
  return y;
}

// Marker of "not yet computed" in the sync-free sweeps: a signalling-NaN bit
// pattern, which IEEE arithmetic never produces (its results are quiet NaNs).
constexpr unsigned long long kPending = 0x7FF0DEAD0BADF00Dull;

// Tunables (mgpu_set_tuning): rows up to which a solve runs in one block, and
// the number of threads taking part in a sync-free triangular sweep.
int g_single_block_rows = 32768;
int g_sweep_threads = 65536;
int g_sweep_sleep = 0;
int g_min_blocks = 1;
}  // namespace
int g_cheb_degree = 24;      // mixed form: Chebyshev-Jacobi degree of the pressure preconditioner
int g_batch_reserve = 0;  // block slots batched launches leave to other streams
int g_prefetch_mb = 96;   // mixed systems whose streamed bytes exceed this prefetch into L2
int prewarm_streams(int n);  // case.cu
double g_cheb_ratio = 1000.0; // and the ratio lambda_max / lambda_min of its interval
// systems of at least g_cheb_large_rows rows (0: none) take the large pair: their
// smallest eigenvalues sit lower, and a wider interval with a higher degree
// pays (3.07 M-tet PISO: 4.50 -> 4.81 steps/s; a 524k channel loses 1-2 %)
int g_cheb_large_rows = 1 << 20;
int g_cheb_degree_large = 48;
double g_cheb_ratio_large = 10000.0;
// the Chebyshev degree and interval ratio of a pressure solve of n rows
void cheb_params(long n, int& k, double& ratio) {
  const bool large = g_cheb_large_rows > 0 && n >= g_cheb_large_rows;
  k = large ? g_cheb_degree_large : g_cheb_degree;
  ratio = large ? g_cheb_ratio_large : g_cheb_ratio;
}
unsigned g_spin_limit = 0; // polls before a bounded barrier wait gives up (0: kSpinLimit, ~2 s)
unsigned g_poll_ns = 100;  // sleep between the polls of a barrier wait (ns)
int g_mixed_occ = 5;       // mixed kernels: resident blocks per SM (2-8; FP64 polynomial 2-5)
int g_gather_faces = 0;    // assembly gathers: faces whose loads a thread issues together (0: per kernel)
int g_batch_occ = 4;       // batched lane kernel: resident blocks per SM (2-5)
namespace {

__device__ __forceinline__ double ld_relaxed_f64(const double* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return __longlong_as_double((long long)v);
}

// Spin (bounded) until p no longer holds kPending; returns the value.
__device__ __forceinline__ double wait_value(const double* p, DevStatus* st, bool& ok, int sleep_ns) {
  double v = ld_relaxed_f64(p);
  unsigned spins = 0;
  while (__double_as_longlong(v) == (long long)kPending) {
    ++spins;
    if ((spins & 1023u) == 0u) {
      if (ld_acquire_i32(&st->timeout) != 0 || spins > (1u << 24)) {
        atomicExch(&st->timeout, 1);
        ok = false;
        return 0.0;
      }
    }
    if (sleep_ns > 0 && spins > 256u) __nanosleep(sleep_ns);
    v = ld_relaxed_f64(p);
  }
  return v;
}

constexpr int kGather = 8;  // dependencies of one row fetched together

// Load x[cols[0..m)] (m <= K) with all loads in flight at once, then re-poll
// only the entries still pending, until none is (bounded).
template <int K>
__device__ __forceinline__ void gather_ready(const double* x, const int* cols, int m, double (&v)[K], DevStatus* st,
                                             bool& ok, int sleep_ns) {
#pragma unroll
  for (int t = 0; t < K; ++t)
    if (t < m) v[t] = ld_relaxed_f64(&x[cols[t]]);
  unsigned spins = 0;
  while (true) {
    bool pend = false;
#pragma unroll
    for (int t = 0; t < K; ++t)
      if (t < m && __double_as_longlong(v[t]) == (long long)kPending) {
        pend = true;
        v[t] = ld_relaxed_f64(&x[cols[t]]);
      }
    if (!pend) return;
    ++spins;
    if ((spins & 1023u) == 0u) {
      if (ld_acquire_i32(&st->timeout) != 0 || spins > (1u << 24)) {
        atomicExch(&st->timeout, 1);
        ok = false;
        return;
      }
    }
    if (sleep_ns > 0 && spins > 256u) __nanosleep(sleep_ns);
  }
}

// A row of a one-block sweep fetched a level ahead: every load that does not
// depend on the previous level's results (the row, its diagonal, the value it
// starts from, its entries' columns and factor values in sweep order) is in
// flight while that level runs, so after the barrier a level waits only for
// its gathers of z. Rows with more than kSweepK entries to apply keep the
// plain loop.
constexpr int kSweepK = 8;
struct SweepRow {
  int i;      // row (-1: none)
  int nk;     // entries to apply
  double s;   // start value: src[i] (forward) or the forward result z[i] (backward)
  double fd;  // f[diag[i]]
  int col[kSweepK];
  double fv[kSweepK];
};

__device__ __forceinline__ void fetch_lo(const KrylovArgs& a, const double* f, const double* src, int idx, int e,
                                         SweepRow& R) {
  R.i = -1;
  if (idx >= e) return;
  const int i = a.lo_rows[idx];
  const int rb = a.row_ptr[i], d = a.diag[i];
  R.i = i;
  R.nk = d - rb;
  R.s = src[i];
  R.fd = f[d];
#pragma unroll
  for (int t = 0; t < kSweepK; ++t)
    if (t < R.nk) {
      R.col[t] = a.col[rb + t];
      R.fv[t] = f[rb + t];
    }
}

__device__ __forceinline__ void fetch_up(const KrylovArgs& a, int kind, const double* f, const double* z, int idx,
                                         int e, SweepRow& R) {
  R.i = -1;
  if (idx >= e) return;
  const int i = a.up_rows[idx];
  const int d = a.diag[i], re = a.row_ptr[i + 1];
  R.i = i;
  R.nk = re - d - 1;
  R.s = z[i];
  R.fd = f[d];
#pragma unroll
  for (int t = 0; t < kSweepK; ++t)
    if (t < R.nk) {
      // IC(0): the L^T entries in descending column order; ILU(0): U ascending
      const int k = kind == 2 ? re - 1 - t : d + 1 + t;
      R.col[t] = a.col[k];
      R.fv[t] = kind == 2 ? f[a.lt_pos[k]] : f[k];
    }
}

// z = M^{-1} src for ILU(0) (kind 0) or IC(0) (kind 2).
// One block: level-scheduled with __syncthreads between levels.
// Several blocks: sync-free. Both sweeps write into arrays pre-filled with
// kPending (forward into a.w, backward into z); each row waits only on the
// entries it reads. Rows are taken in level order and every thread walks its
// rows in that order, so the lowest unfinished row can always proceed: all
// blocks being co-resident, the sweep completes. The arithmetic of each row is
// the reference's, in the reference's order.
template <bool L1>
__device__ bool apply_lu(const KrylovArgs& a, int kind, const double* src, double* z) {
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstr = gridDim.x * blockDim.x;
  const double* f = a.fval;
  if constexpr (L1) {
    SweepRow R;
    R.i = -1;
    if (a.nlev_lo > 0) fetch_lo(a, f, src, a.lo_ptr[0] + gtid, a.lo_ptr[1], R);
    for (int lev = 0; lev < a.nlev_lo; ++lev) {
      const int e = a.lo_ptr[lev + 1];
      if (R.i >= 0) {  // this thread's first row of the level, fetched ahead
        double s = R.s;
        if (R.nk <= kSweepK) {
#pragma unroll
          for (int t = 0; t < kSweepK; ++t)
            if (t < R.nk) s = s - R.fv[t] * z[R.col[t]];
        } else {
          for (int k = a.row_ptr[R.i]; k < a.diag[R.i]; ++k) s = s - f[k] * z[a.col[k]];
        }
        z[R.i] = (kind == 2) ? s / R.fd : s;
      }
      for (int idx = a.lo_ptr[lev] + gtid + gstr; idx < e; idx += gstr) {
        const int i = a.lo_rows[idx];
        double s = src[i];
        const int d = a.diag[i];
        for (int k = a.row_ptr[i]; k < d; ++k) s = s - f[k] * z[a.col[k]];
        z[i] = (kind == 2) ? s / f[d] : s;
      }
      if (lev + 1 < a.nlev_lo) fetch_lo(a, f, src, e + gtid, a.lo_ptr[lev + 2], R);
      __syncthreads();
    }
    // the forward results are final here: a backward row's start value z[i]
    // is only rewritten in its own level, so it may be fetched a level ahead
    R.i = -1;
    if (a.nlev_up > 0) fetch_up(a, kind, f, z, a.up_ptr[0] + gtid, a.up_ptr[1], R);
    for (int lev = 0; lev < a.nlev_up; ++lev) {
      const int e = a.up_ptr[lev + 1];
      if (R.i >= 0) {
        double s = R.s;
        if (R.nk <= kSweepK) {
#pragma unroll
          for (int t = 0; t < kSweepK; ++t)
            if (t < R.nk) s = s - R.fv[t] * z[R.col[t]];
        } else {
          const int d = a.diag[R.i], re = a.row_ptr[R.i + 1];
          if (kind == 2) {
            for (int k = re - 1; k > d; --k) s = s - f[a.lt_pos[k]] * z[a.col[k]];
          } else {
            for (int k = d + 1; k < re; ++k) s = s - f[k] * z[a.col[k]];
          }
        }
        z[R.i] = s / R.fd;
      }
      for (int idx = a.up_ptr[lev] + gtid + gstr; idx < e; idx += gstr) {
        const int i = a.up_rows[idx];
        const int d = a.diag[i], re = a.row_ptr[i + 1];
        double s = z[i];
        if (kind == 2) {
          // L^T z = y, column sweep of ic0_apply: w(i) collects -L(j,i) z(j)
          // for j = n..i+1 (descending), then z(i) = w(i)/L(i,i).
          for (int k = re - 1; k > d; --k) s = s - f[a.lt_pos[k]] * z[a.col[k]];
        } else {
          for (int k = d + 1; k < re; ++k) s = s - f[k] * z[a.col[k]];
        }
        z[i] = s / f[d];
      }
      if (lev + 1 < a.nlev_up) fetch_up(a, kind, f, z, e + gtid, a.up_ptr[lev + 2], R);
      __syncthreads();
    }
    return true;
  } else {
    const int n = a.n;
    double* y = a.w;
    const double pend = __longlong_as_double((long long)kPending);
    for (int i = gtid; i < n; i += gstr) {
      y[i] = pend;
      z[i] = pend;
    }
    if (!grid_sync(a.bar, a.st)) return false;
    bool ok = true;
    const int P = gstr < a.sweep_threads ? gstr : a.sweep_threads;
    const int sl = a.sweep_sleep;
    if (gtid < P) {
      for (int idx = gtid; idx < n && ok; idx += P) {
        const int i = a.lo_rows[idx];
        const int rb = a.row_ptr[i], d = a.diag[i];
        double s = ldv(&src[i]);
        if (d - rb <= kGather) {
          double v[kGather];
          gather_ready<kGather>(y, a.col + rb, d - rb, v, a.st, ok, sl);
#pragma unroll
          for (int t = 0; t < kGather; ++t)
            if (t < d - rb) s = s - f[rb + t] * v[t];
        } else {
          for (int k = rb; k < d && ok; ++k) s = s - f[k] * wait_value(&y[a.col[k]], a.st, ok, sl);
        }
        __stcg(&y[i], (kind == 2) ? s / f[d] : s);
      }
      for (int idx = gtid; idx < n && ok; idx += P) {
        const int i = a.up_rows[idx];
        const int d = a.diag[i], re = a.row_ptr[i + 1];
        const int nu = re - d - 1;
        double s = wait_value(&y[i], a.st, ok, sl);
        if (nu <= kGather) {
          double v[kGather];
          gather_ready<kGather>(z, a.col + d + 1, nu, v, a.st, ok, sl);
          if (kind == 2) {
            // descending column order (ic0_apply's Lt sweep)
#pragma unroll
            for (int t = kGather - 1; t >= 0; --t)
              if (t < nu) s = s - f[a.lt_pos[d + 1 + t]] * v[t];
          } else {
#pragma unroll
            for (int t = 0; t < kGather; ++t)
              if (t < nu) s = s - f[d + 1 + t] * v[t];
          }
        } else if (kind == 2) {
          for (int k = re - 1; k > d && ok; --k) s = s - f[a.lt_pos[k]] * wait_value(&z[a.col[k]], a.st, ok, sl);
        } else {
          for (int k = d + 1; k < re && ok; ++k) s = s - f[k] * wait_value(&z[a.col[k]], a.st, ok, sl);
        }
        __stcg(&z[i], s / f[d]);
      }
    }
    return grid_sync(a.bar, a.st);
  }
}

__device__ void write_result(const KrylovArgs& a, int it, double res, int ierr) {
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


// ---------------------------------------------------------------------------
// Factorisation kernel: ILU(0) (kind 0) or IC(0) (kind 2) of aval into fval.
// ---------------------------------------------------------------------------
template <bool L1>
__global__ void __launch_bounds__(L1 ? 512 : 256) k_factor(KrylovArgs a, int kind) {
  if (a.st->abort) return;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstr = gridDim.x * blockDim.x;
  if (gtid == 0) *a.ferr = 0;
  const int nnz = a.row_ptr[a.n];
  for (int k = gtid; k < nnz; k += gstr) a.fval[k] = a.aval[k];
  if (!grid_sync(a.bar, a.st)) return;
  double* f = a.fval;
  for (int lev = 0; lev < a.nlev_lo; ++lev) {
    const int e = a.lo_ptr[lev + 1];
    for (int idx = a.lo_ptr[lev] + gtid; idx < e; idx += gstr) {
      const int i = a.lo_rows[idx];
      const int rb = a.row_ptr[i], re = a.row_ptr[i + 1], di = a.diag[i];
      if (kind == 0) {
        // ilu0_factor row i (IKJ): rows k < i are final
        for (int kk = rb; kk < di; ++kk) {
          const int k = a.col[kk];
          const double piv = ldv(&f[a.diag[k]]);
          if (fabs(piv) < DTINY) {
            atomicExch(a.ferr, 2);
            continue;
          }
          const double aik = f[kk] / piv;
          f[kk] = aik;
          int pos = kk + 1;  // merge pointer into row i (columns ascending)
          const int ke = a.row_ptr[k + 1];
          for (int jj = a.diag[k]; jj < ke; ++jj) {
            const int j = a.col[jj];
            if (j <= k) continue;
            while (pos < re && a.col[pos] < j) ++pos;
            if (pos < re && a.col[pos] == j) f[pos] = f[pos] - aik * ldv(&f[jj]);
          }
        }
      } else {
        // ic0_factor row i
        for (int kp = rb; kp < di; ++kp) {
          const int k = a.col[kp];
          // ic0_dot(row i [rb, kp-1], row k [row_ptr(k), diag(k)-1])
          int p = rb, q = a.row_ptr[k];
          const int p2 = kp - 1, q2 = a.diag[k] - 1;
          double dsum = 0.0;
          while (p <= p2 && q <= q2) {
            const int cp = a.col[p], cq = a.col[q];
            if (cp < cq)
              ++p;
            else if (cp > cq)
              ++q;
            else {
              dsum = dsum + f[p] * ldv(&f[q]);
              ++p;
              ++q;
            }
          }
          const double s = f[kp] - dsum;
          f[kp] = s / ldv(&f[a.diag[k]]);
        }
        double s = f[di];
        for (int kp = rb; kp < di; ++kp) s = s - f[kp] * f[kp];
        if (s <= 0.0) atomicExch(a.ferr, 2);
        f[di] = sqrt(s);
      }
    }
    if (!grid_sync(a.bar, a.st)) return;
  }
}

// ---------------------------------------------------------------------------
// PCG: cg_jacobi / cg_ic0 (and PCG with ILU(0)); `it` ends at maxit+1 on
// non-convergence, as the Fortran DO loop leaves it.
// ---------------------------------------------------------------------------
template <bool L1>
__global__ void __launch_bounds__(L1 ? 512 : 256) k_pcg(KrylovArgs a) {
  if (a.st->abort) return;
  const int n = a.n;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstr = gridDim.x * blockDim.x;
  VGrid vg = whole_grid(a.bar, a.partials);
  const bool jac = a.precond == 1;
  double* x = a.x;
  double *r = a.r, *z = a.z, *p = a.p, *q = a.v;
  // b.b and (Jacobi, one-rank distributed form) the count of |diag| < tiny
  double v2[2] = {0.0, 0.0};
  for (int i = gtid; i < n; i += gstr) {
    if (a.zero_x) x[i] = 0.0;
    const double bi = a.b[i];
    v2[0] = v2[0] + bi * bi;
    if (jac && fabs(a.aval[a.diag[i]]) < DTINY) v2[1] = v2[1] + 1.0;
  }
  if (!vg_sum<2, L1>(v2, vg, a.st)) return;
  const double bnrm = sqrt(v2[0]);
  if (bnrm == 0.0) {
    for (int i = gtid; i < n; i += gstr) x[i] = 0.0;
    write_result(a, 0, 0.0, 0);
    return;
  }
  if (!jac && *a.ferr != 0) {
    write_result(a, 0, 0.0, *a.ferr + 10);
    return;
  }
  if (jac && v2[1] != 0.0 && a.mpi_mode) {  // cg_jacobi_mpi rejects |diag| < tiny
    write_result(a, 0, 0.0, 2);
    return;
  }
  // r = b - A x ; (Jacobi) z = r/diag
  double w2[2] = {0.0, 0.0};
  for (int i = gtid; i < n; i += gstr) {
    const double ri = a.b[i] - row_spmv<L1>(a.row_ptr, a.col, a.aval, x, i);
    r[i] = ri;
    w2[0] = w2[0] + ri * ri;
    if (jac) {
      const double zi = ri / a.aval[a.diag[i]];
      z[i] = zi;
      w2[1] = w2[1] + ri * zi;
    }
  }
  if (!vg_sum<2, L1>(w2, vg, a.st)) return;
  double res = sqrt(w2[0]) / bnrm;
  if (res <= a.tol) {
    write_result(a, 0, res, 0);
    return;
  }
  double rz;
  if (jac) {
    rz = w2[1];
  } else {
    if (!apply_lu<L1>(a, a.precond, r, z)) return;
    double v1[1] = {0.0};
    for (int i = gtid; i < n; i += gstr) v1[0] = v1[0] + r[i] * ldv(&z[i]);
    if (!vg_sum<1, L1>(v1, vg, a.st)) return;
    rz = v1[0];
  }
  for (int i = gtid; i < n; i += gstr) p[i] = ldv(&z[i]);
  if (!grid_sync(a.bar, a.st)) return;
  int ierr = 0, it;
  for (it = 1; it <= a.maxit; ++it) {
    double pq[1] = {0.0};
    for (int i = gtid; i < n; i += gstr) {
      const double qi = row_spmv<L1>(a.row_ptr, a.col, a.aval, p, i);
      q[i] = qi;
      pq[0] = pq[0] + p[i] * qi;
    }
    if (!vg_sum<1, L1>(pq, vg, a.st)) return;
    const double pap = pq[0];
    if (fabs(pap) < DTINY) {
      ierr = 2;
      break;
    }
    const double alpha = rz / pap;
    double u2[2] = {0.0, 0.0};
    for (int i = gtid; i < n; i += gstr) {
      x[i] = x[i] + alpha * p[i];
      const double ri = r[i] - alpha * q[i];
      r[i] = ri;
      u2[0] = u2[0] + ri * ri;
      if (jac) {
        const double zi = ri / a.aval[a.diag[i]];
        z[i] = zi;
        u2[1] = u2[1] + ri * zi;
      }
    }
    if (!vg_sum<2, L1>(u2, vg, a.st)) return;
    res = sqrt(u2[0]) / bnrm;
    if (res <= a.tol) {
      write_result(a, it, res, 0);
      return;
    }
    double rz_new;
    if (jac) {
      rz_new = u2[1];
    } else {
      if (!apply_lu<L1>(a, a.precond, r, z)) return;
      double v1[1] = {0.0};
      for (int i = gtid; i < n; i += gstr) v1[0] = v1[0] + r[i] * ldv(&z[i]);
      if (!vg_sum<1, L1>(v1, vg, a.st)) return;
      rz_new = v1[0];
    }
    if (fabs(rz) < DTINY) {
      ierr = 2;
      break;
    }
    const double beta = rz_new / rz;
    for (int i = gtid; i < n; i += gstr) p[i] = ldv(&z[i]) + beta * p[i];
    if (!grid_sync(a.bar, a.st)) return;
    rz = rz_new;
  }
  if (ierr == 0) ierr = 1;
  write_result(a, it, res, ierr);
}

// ---------------------------------------------------------------------------
// BiCGStab, right-preconditioned with ILU(0) (bicgstab_ilu0) or Jacobi.
// ---------------------------------------------------------------------------
template <bool L1>
__global__ void __launch_bounds__(L1 ? 512 : 256) k_bicgstab(KrylovArgs a) {
  if (a.st->abort) return;
  const int n = a.n;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstr = gridDim.x * blockDim.x;
  VGrid vg = whole_grid(a.bar, a.partials);
  const bool jac = a.precond == 1;
  double* x = a.x;
  double *r = a.r, *r0 = a.r0, *p = a.p, *v = a.v, *s = a.s, *t = a.t, *ph = a.ph, *sh = a.sh;
  double v2[2] = {0.0, 0.0};
  for (int i = gtid; i < n; i += gstr) {
    const double bi = a.b[i];
    v2[0] = v2[0] + bi * bi;
    if (jac && fabs(a.aval[a.diag[i]]) < DTINY) v2[1] = v2[1] + 1.0;
  }
  if (!vg_sum<2, L1>(v2, vg, a.st)) return;
  const double bnrm = sqrt(v2[0]);
  if (bnrm == 0.0) {
    for (int i = gtid; i < n; i += gstr) x[i] = 0.0;
    write_result(a, 0, 0.0, 0);
    return;
  }
  if (!jac && *a.ferr != 0) {
    write_result(a, 0, 0.0, *a.ferr + 10);
    return;
  }
  if (jac && v2[1] != 0.0) {
    write_result(a, 0, 0.0, 12);
    return;
  }
  double w1[1] = {0.0};
  for (int i = gtid; i < n; i += gstr) {
    const double ri = a.b[i] - row_spmv<L1>(a.row_ptr, a.col, a.aval, x, i);
    r0[i] = ri;
    r[i] = ri;
    p[i] = 0.0;
    v[i] = 0.0;
    w1[0] = w1[0] + ri * ri;
  }
  if (!vg_sum<1, L1>(w1, vg, a.st)) return;
  double res = sqrt(w1[0]) / bnrm;
  if (res <= a.tol) {
    write_result(a, 0, res, 0);
    return;
  }
  double rho_next = w1[0];  // dot(r, r0) with r == r0: the same sum as r0.r0
  double rho_old = 1.0, alpha = 1.0, omega = 1.0;
  int ierr = 0, it;
  for (it = 1; it <= a.maxit; ++it) {
    const double rho = rho_next;
    if (fabs(rho) < DTINY) {
      ierr = 2;
      break;
    }
    const double beta = (rho / rho_old) * (alpha / omega);
    for (int i = gtid; i < n; i += gstr) {
      const double pi = r[i] + beta * (p[i] - omega * v[i]);
      p[i] = pi;
      if (jac) ph[i] = pi / a.aval[a.diag[i]];
    }
    if (!grid_sync(a.bar, a.st)) return;
    if (!jac && !apply_lu<L1>(a, 0, p, ph)) return;
    double d1[1] = {0.0};
    for (int i = gtid; i < n; i += gstr) {
      const double vi = row_spmv<L1>(a.row_ptr, a.col, a.aval, ph, i);
      v[i] = vi;
      d1[0] = d1[0] + r0[i] * vi;
    }
    if (!vg_sum<1, L1>(d1, vg, a.st)) return;
    alpha = rho / d1[0];
    double d2[1] = {0.0};
    for (int i = gtid; i < n; i += gstr) {
      const double si = r[i] - alpha * v[i];
      s[i] = si;
      d2[0] = d2[0] + si * si;
      if (jac) sh[i] = si / a.aval[a.diag[i]];
    }
    if (!vg_sum<1, L1>(d2, vg, a.st)) return;
    const double snrm = sqrt(d2[0]);
    if (snrm / bnrm <= a.tol) {
      for (int i = gtid; i < n; i += gstr) x[i] = x[i] + alpha * ldv(&ph[i]);
      write_result(a, it, snrm / bnrm, 0);
      return;
    }
    if (!jac && !apply_lu<L1>(a, 0, s, sh)) return;
    double d3[2] = {0.0, 0.0};
    for (int i = gtid; i < n; i += gstr) {
      const double ti = row_spmv<L1>(a.row_ptr, a.col, a.aval, sh, i);
      t[i] = ti;
      d3[0] = d3[0] + ti * ti;
      d3[1] = d3[1] + ti * s[i];
    }
    if (!vg_sum<2, L1>(d3, vg, a.st)) return;
    const double tt = d3[0];
    if (tt < DTINY) {
      ierr = 2;
      break;
    }
    omega = d3[1] / tt;
    if (fabs(omega) < DTINY) {
      ierr = 2;
      break;
    }
    double d4[2] = {0.0, 0.0};
    for (int i = gtid; i < n; i += gstr) {
      x[i] = x[i] + alpha * ldv(&ph[i]) + omega * ldv(&sh[i]);
      const double ri = s[i] - omega * t[i];
      r[i] = ri;
      d4[0] = d4[0] + ri * ri;
      d4[1] = d4[1] + ri * r0[i];
    }
    if (!vg_sum<2, L1>(d4, vg, a.st)) return;
    res = sqrt(d4[0]) / bnrm;
    if (res <= a.tol) {
      write_result(a, it, res, 0);
      return;
    }
    rho_next = d4[1];
    rho_old = rho;
  }
  if (ierr == 0) {
    ierr = 1;
    it = a.maxit;
  }
  write_result(a, it, res, ierr);
}

__global__ void k_spmv(int n, const int* __restrict__ rp, const int* __restrict__ col,
                       const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  const int e = rp[i + 1];
  for (int k = rp[i]; k < e; ++k) s = s + val[k] * x[col[k]];
  y[i] = s;
}

int launch_coop(const void* fn, void** args, unsigned long long* bar, int grid, int block, cudaStream_t s,
                bool coop) {
  cudaError_t e = cudaMemsetAsync(bar, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return cuda_fail(e, "barrier reset", __FILE__, __LINE__);
  if (coop)
    e = cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(block), args, 0, s);
  else
    e = cudaLaunchKernel(fn, dim3(grid), dim3(block), args, 0, s);
  if (e != cudaSuccess) return cuda_fail(e, "cooperative launch", __FILE__, __LINE__);
  return 0;
}

}  // namespace

// Grid of a persistent Krylov kernel: one 512-thread block (single-SM mode,
// no grid barrier) for small systems, else enough 256-thread blocks for ~4
// rows per thread, capped by co-residency.
int krylov_grid(int n, int& block, int which) {
  constexpr int kDevs = 64;  // co-resident capacity, per device (GPUs of a node may differ)
  static int max_blocks[kDevs][3] = {};
  if (n <= g_single_block_rows) {
    block = 512;
    return 1;
  }
  block = 256;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kDevs) dev = 0;
  int (&mb)[3] = max_blocks[dev];
  if (mb[which] == 0) {
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const void* fn = which == 0 ? (const void*)k_pcg<false>
                                : which == 1 ? (const void*)k_bicgstab<false> : (const void*)k_factor<false>;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, block, 0);
    if (per < 1) per = 1;
    mb[which] = sms * per;
  }
  long want = ((long)n + (long)block * 4 - 1) / ((long)block * 4);
  if (want < g_min_blocks) want = g_min_blocks;
  if (want < 1) want = 1;
  if (want > mb[which]) want = mb[which];
  return (int)want;
}

int launch_krylov_pcg(const KrylovArgs& a, cudaStream_t s) {
  int block = 0;
  const int grid = krylov_grid(a.n, block, 0);
  KrylovArgs aa = a;
  aa.sweep_threads = g_sweep_threads;
  aa.sweep_sleep = g_sweep_sleep;
  void* args[] = {&aa};
  return launch_coop(grid == 1 ? (const void*)k_pcg<true> : (const void*)k_pcg<false>, args, a.bar, grid, block, s,
                     true);
}

int launch_krylov_bicgstab(const KrylovArgs& a, cudaStream_t s) {
  int block = 0;
  const int grid = krylov_grid(a.n, block, 1);
  KrylovArgs aa = a;
  aa.sweep_threads = g_sweep_threads;
  aa.sweep_sleep = g_sweep_sleep;
  void* args[] = {&aa};
  return launch_coop(grid == 1 ? (const void*)k_bicgstab<true> : (const void*)k_bicgstab<false>, args, a.bar, grid,
                     block, s, true);
}

int launch_factor(const KrylovArgs& a, int kind, cudaStream_t s) {
  int block = 0;
  const int grid = krylov_grid(a.n, block, 2);
  KrylovArgs aa = a;
  int kk = kind;
  void* args[] = {&aa, &kk};
  return launch_coop(grid == 1 ? (const void*)k_factor<true> : (const void*)k_factor<false>, args, a.bar, grid, block,
                     s, true);
}

int launch_spmv(int n, const int* rp, const int* col, const double* val, const double* x, double* y,
                cudaStream_t s) {
  k_spmv<<<ceil_div(n, 256), 256, 0, s>>>(n, rp, col, val, x, y);
  MGPU_LAUNCH_CHECK("k_spmv");
  return 0;
}

int set_tuning(const char* key, int value) {
  const std::string k(key ? key : "");
  if (k == "single_block_rows" && value >= 0) {
    g_single_block_rows = value;
  } else if (k == "sweep_threads" && value >= 32) {
    g_sweep_threads = value;
  } else if (k == "cheb_degree" && value >= 1 && value <= 64) {
    g_cheb_degree = value;
  } else if (k == "cheb_ratio" && value >= 2) {
    g_cheb_ratio = value;
  } else if (k == "cheb_large_rows" && value >= 0) {
    g_cheb_large_rows = value;
  } else if (k == "cheb_degree_large" && value >= 1 && value <= 64) {
    g_cheb_degree_large = value;
  } else if (k == "cheb_ratio_large" && value >= 2) {
    g_cheb_ratio_large = value;
  } else if (k == "min_blocks" && value >= 1) {
    g_min_blocks = value;
  } else if (k == "sweep_sleep_ns" && value >= 0 && value <= 100000) {
    g_sweep_sleep = value;
  } else if (k == "batch_reserve_blocks" && value >= 0 && value <= 256) {
    g_batch_reserve = value;
  } else if (k == "l2_prefetch_mb" && value >= 0) {
    g_prefetch_mb = value;
  } else if (k == "mixed_blocks_per_sm" && value >= 2 && value <= 8) {
    g_mixed_occ = value;
  } else if (k == "batch_blocks_per_sm" && value >= 2 && value <= 5) {
    g_batch_occ = value;
  } else if (k == "spin_limit" && value >= 0) {
    g_spin_limit = (unsigned)value;
  } else if (k == "gather_faces" && value >= 0 && value <= 6) {
    g_gather_faces = value;
  } else if (k == "barrier_poll_ns" && value >= 0 && value <= 10000) {
    g_poll_ns = (unsigned)value;
  } else if (k == "stream_pool" && value >= 0 && value <= 1024) {
    if (int e = prewarm_streams(value)) return e;
  } else {
    set_error("mgpu_set_tuning: unknown key or value out of range: " + k);
    return MGPU_E_ARG;
  }
  return 0;
}

int get_tuning(const char* key, int* value) {
  const std::string k(key ? key : "");
  if (!value) return MGPU_E_ARG;
  if (k == "single_block_rows") {
    *value = g_single_block_rows;
  } else if (k == "sweep_threads") {
    *value = g_sweep_threads;
  } else if (k == "cheb_degree") {
    *value = g_cheb_degree;
  } else if (k == "cheb_ratio") {
    *value = (int)g_cheb_ratio;
  } else if (k == "cheb_large_rows") {
    *value = g_cheb_large_rows;
  } else if (k == "cheb_degree_large") {
    *value = g_cheb_degree_large;
  } else if (k == "cheb_ratio_large") {
    *value = (int)g_cheb_ratio_large;
  } else if (k == "min_blocks") {
    *value = g_min_blocks;
  } else if (k == "sweep_sleep_ns") {
    *value = g_sweep_sleep;
  } else if (k == "batch_reserve_blocks") {
    *value = g_batch_reserve;
  } else if (k == "l2_prefetch_mb") {
    *value = g_prefetch_mb;
  } else if (k == "mixed_blocks_per_sm") {
    *value = g_mixed_occ;
  } else if (k == "batch_blocks_per_sm") {
    *value = g_batch_occ;
  } else if (k == "spin_limit") {
    *value = (int)g_spin_limit;
  } else if (k == "gather_faces") {
    *value = g_gather_faces;
  } else if (k == "barrier_poll_ns") {
    *value = (int)g_poll_ns;
  } else {
    set_error("mgpu_get_tuning: unknown key: " + k);
    return MGPU_E_ARG;
  }
  return 0;
}

}  // namespace mgpu

extern "C" int mgpu_set_tuning(const char* key, int value) { return mgpu::set_tuning(key, value); }
extern "C" int mgpu_get_tuning(const char* key, int* value) { return mgpu::get_tuning(key, value); }
