// standalone.cu -- C-ABI entry points that work on plain host arrays:
// Krylov solves and SpMV on a CSR matrix (the mod_uns_linsolver interface),
// and the mesh pipeline (connectivity, geometry, RCM ordering).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "assembly.cuh"
#include "case.cuh"
#include "device_topo.h"
#include "mesh_host.h"

namespace mgpu {
extern unsigned g_spin_limit;  // krylov.cu: the spin_limit tuning key
extern unsigned g_poll_ns;     // krylov.cu: the barrier_poll_ns tuning key
extern int g_cheb_degree;      // the cheb_degree and cheb_ratio tuning keys
extern double g_cheb_ratio;
void cheb_params(long n, int& k, double& ratio);  // krylov.cu
extern int g_prefetch_mb;      // l2_prefetch_mb
}

using namespace mgpu;

namespace {

struct DevBuf {
  std::vector<void*> p;
  ~DevBuf() {
    for (void* q : p) cudaFree(q);
  }
  template <typename T>
  int alloc(T*& out, size_t n) {
    void* q = nullptr;
    MGPU_CUDA(cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T)));
    p.push_back(q);
    out = (T*)q;
    return 0;
  }
  template <typename T>
  int up(T*& out, const T* h, size_t n) {
    if (int e = alloc(out, n)) return e;
    if (n) MGPU_CUDA(cudaMemcpy(out, h, n * sizeof(T), cudaMemcpyHostToDevice));
    return 0;
  }
};

#define TRY(x)                 \
  do {                         \
    int rc_ = (x);             \
    if (rc_ != 0) return rc_;  \
  } while (0)

// Level sets / transposes of an arbitrary CSR pattern (0-based).
struct Pattern {
  std::vector<int> rp, col, diag, mirror, lo_ptr, lo_rows, up_ptr, up_rows;
  int nlo = 0, nup = 0;
  bool symmetric = true, full_diag = true;
};

void analyse(int n, const int32_t* row_ptr, const int32_t* col_idx, Pattern& P) {
  P.rp.resize(n + 1);
  for (int i = 0; i <= n; ++i) P.rp[i] = row_ptr[i] - 1;
  const int nnz = P.rp[n];
  P.col.resize(nnz);
  for (int k = 0; k < nnz; ++k) P.col[k] = col_idx[k] - 1;
  auto find = [&](int i, int j) {
    for (int k = P.rp[i]; k < P.rp[i + 1]; ++k) {
      if (P.col[k] == j) return k;
      if (P.col[k] > j) return -1;
    }
    return -1;
  };
  P.diag.resize(n);
  for (int i = 0; i < n; ++i) {
    P.diag[i] = find(i, i);
    if (P.diag[i] < 0) P.full_diag = false;
  }
  P.mirror.assign(nnz, 0);
  for (int i = 0; i < n; ++i)
    for (int k = P.rp[i]; k < P.rp[i + 1]; ++k) {
      P.mirror[k] = find(P.col[k], i);
      if (P.mirror[k] < 0) {
        P.symmetric = false;
        P.mirror[k] = k;
      }
    }
  if (!P.full_diag) return;
  std::vector<int> lev(n, 0);
  for (int i = 0; i < n; ++i) {
    int l = 0;
    for (int k = P.rp[i]; k < P.diag[i]; ++k) l = std::max(l, lev[P.col[k]] + 1);
    lev[i] = l;
    P.nlo = std::max(P.nlo, l + 1);
  }
  auto bucket = [&](int nl, std::vector<int>& ptr, std::vector<int>& rows) {
    ptr.assign(nl + 1, 0);
    for (int i = 0; i < n; ++i) ptr[lev[i] + 1]++;
    for (int l = 0; l < nl; ++l) ptr[l + 1] += ptr[l];
    rows.assign(n, 0);
    std::vector<int> f(ptr.begin(), ptr.end() - 1);
    for (int i = 0; i < n; ++i) rows[f[lev[i]]++] = i;
  };
  bucket(P.nlo, P.lo_ptr, P.lo_rows);
  for (int i = n - 1; i >= 0; --i) {
    int l = 0;
    for (int k = P.diag[i] + 1; k < P.rp[i + 1]; ++k) l = std::max(l, lev[P.col[k]] + 1);
    lev[i] = l;
    P.nup = std::max(P.nup, l + 1);
  }
  bucket(P.nup, P.up_ptr, P.up_rows);
}

// The pressure solver of the mixed and FP64 polynomial forms on a host CSR
// system: the case's own kernels (k_pcg_mixed / k_pcg_poly64) with the
// arguments a case would give them, the ELL copy built on the device.
template <typename V>
int poly_solve(int n, const Pattern& P, const double* val, const double* b, double* x, double tol, int maxit,
                      int cheb_degree, double cheb_ratio, int* it, double* res, int* ierr) {
  DevBuf B;
  const int nnz = P.rp[n];
  int *drp, *dcol, *ddiag, *dferr;
  double *dval, *db, *dx, *dkw, *dpart, *dred;
  V *da, *ddinv, *dw;
  unsigned long long* dbar;
  DevStatus* dst;
  MgpuIterRec* drec;
  TRY(B.up(drp, P.rp.data(), n + 1));
  TRY(B.up(dcol, P.col.data(), nnz));
  TRY(B.up(ddiag, P.diag.data(), n));
  TRY(B.up(dval, val, nnz));
  TRY(B.up(db, b, n));
  TRY(B.up(dx, x, n));
  TRY(B.alloc(dkw, 10 * (size_t)n));
  TRY(B.alloc(dpart, 4 * 4096));
  TRY(B.alloc(dred, (size_t)mixed_red_words(n)));
  TRY(B.alloc(da, nnz));
  TRY(B.alloc(ddinv, n));
  TRY(B.alloc(dw, 10 * (size_t)n));
  TRY(B.alloc(dbar, 1));
  TRY(B.alloc(dferr, 1));
  TRY(B.alloc(dst, 1));
  TRY(B.alloc(drec, 1));
  int W = 0, *ell = nullptr;
  long ld = 0;
  TopoAlloc alloc = [&](int*& q, size_t k) { return B.alloc(q, k); };
  TRY(device_ell(n, drp, dcol, 8, W, ld, ell, alloc, 0));
  V* dev = nullptr;
  double* dev64 = nullptr;  // the mixed form's FP64 conjugate-gradient product
  if (ell) {
    TRY(B.alloc(dev, (size_t)W * ld));
    MGPU_CUDA(cudaMemset(dev, 0, sizeof(V) * (size_t)W * ld));
    if (sizeof(V) == 4) {
      TRY(B.alloc(dev64, (size_t)W * ld));
      MGPU_CUDA(cudaMemset(dev64, 0, sizeof(double) * (size_t)W * ld));
    }
  }
  DevStatus h{};
  h.nan_key = ~0ull;
  h.spin_limit = g_spin_limit;
  h.poll_ns = g_poll_ns;
  MGPU_CUDA(cudaMemcpy(dst, &h, sizeof(h), cudaMemcpyHostToDevice));
  MGPU_CUDA(cudaMemset(drec, 0, sizeof(MgpuIterRec)));
  KrylovArgs a{};
  a.n = n;
  a.row_ptr = drp;
  a.col = dcol;
  a.diag = ddiag;
  a.aval = dval;
  a.b = db;
  a.x = dx;
  a.r = dkw;
  a.p = dkw + 2l * n;
  a.v = dkw + 3l * n;
  a.s = dkw + 4l * n;
  a.tol = tol;
  a.maxit = maxit;
  a.precond = 1;
  a.partials = dpart;
  a.bar = dbar;
  a.st = dst;
  a.recs = drec;
  a.ferr = dferr;
  const bool mixed = sizeof(V) == 4;
  const double row_bytes = mixed ? mixed_row_bytes(W) : 16.0 * W + 80.0;
  const bool big = (double)n * row_bytes > g_prefetch_mb * 1048576.0;
  MixedArgsT<V> m{da,   ddinv, dw, 1e-4, cheb_degree, cheb_ratio, W, ell, dev, dred, (ell && big) ? 1 : 0, 0.0,
                  (int)ld, 0,  dev64};
  if constexpr (sizeof(V) == 4)
    TRY(launch_pcg_mixed(a, m, 0));
  else
    TRY(launch_pcg_poly64(a, m, 0));
  MGPU_CUDA(cudaDeviceSynchronize());
  MgpuIterRec r{};
  MGPU_CUDA(cudaMemcpy(&r, drec, sizeof(r), cudaMemcpyDeviceToHost));
  MGPU_CUDA(cudaMemcpy(&h, dst, sizeof(h), cudaMemcpyDeviceToHost));
  MGPU_CUDA(cudaMemcpy(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (h.timeout) {
    set_error("a bounded device wait ran out (grid barrier)");
    return MGPU_E_TIMEOUT;
  }
  *it = r.lin_it[0];
  *res = r.lin_res[0];
  *ierr = r.lin_ierr[0];
  return 0;
}

}  // namespace

extern "C" {

int mgpu_krylov_solve(int n, const int32_t* row_ptr, const int32_t* col_idx, const double* val, const double* b,
                      double* x, double tol, int maxit, int method, int norm_mode, int* it, double* res,
                      int* ierr) {
  if (n <= 0 || !row_ptr || !col_idx || !val || !b || !x || !it || !res || !ierr || method < 0 || method > 4 ||
      maxit < 0) {
    set_error("mgpu_krylov_solve: invalid argument");
    return MGPU_E_ARG;
  }
  Pattern P;
  analyse(n, row_ptr, col_idx, P);
  const int precond = (method == 0 || method == 4) ? 0 : (method == 2 ? 2 : 1);
  const bool bicg = method == 0 || method == 3;
  *it = 0;
  *res = 0.0;
  *ierr = 0;
  if (!P.full_diag) {
    // the reference checks b = 0 first, then the missing diagonal
    bool bz = true;
    for (int i = 0; i < n; ++i) bz = bz && (b[i] == 0.0);
    if (bz) {
      for (int i = 0; i < n; ++i) x[i] = 0.0;
      return 0;
    }
    *ierr = (precond == 1) ? (bicg ? 12 : 2) : 11;
    return 0;
  }
  if (precond == 2 && !P.symmetric) {
    set_error("mgpu_krylov_solve: IC(0) needs a structurally symmetric pattern");
    return MGPU_E_ARG;
  }
  DevBuf B;
  const int nnz = P.rp[n];
  int *drp, *dcol, *ddiag, *dmir, *dlop, *dlor, *dupp, *dupr, *dferr;
  double *dval, *dfval, *db, *dx, *dkw, *dpart;
  unsigned long long* dbar;
  DevStatus* dst;
  MgpuIterRec* drec;
  TRY(B.up(drp, P.rp.data(), n + 1));
  TRY(B.up(dcol, P.col.data(), nnz));
  TRY(B.up(ddiag, P.diag.data(), n));
  TRY(B.up(dmir, P.mirror.data(), nnz));
  TRY(B.up(dlop, P.lo_ptr.data(), P.lo_ptr.size()));
  TRY(B.up(dlor, P.lo_rows.data(), n));
  TRY(B.up(dupp, P.up_ptr.data(), P.up_ptr.size()));
  TRY(B.up(dupr, P.up_rows.data(), n));
  TRY(B.up(dval, val, nnz));
  TRY(B.alloc(dfval, nnz));
  TRY(B.up(db, b, n));
  TRY(B.up(dx, x, n));
  TRY(B.alloc(dkw, 10 * (size_t)n));
  TRY(B.alloc(dpart, 4 * 4096));
  TRY(B.alloc(dbar, 1));
  TRY(B.alloc(dferr, 1));
  TRY(B.alloc(dst, 1));
  TRY(B.alloc(drec, 1));
  DevStatus h{};
  h.nan_key = ~0ull;
  h.spin_limit = g_spin_limit;
  h.poll_ns = g_poll_ns;
  MGPU_CUDA(cudaMemcpy(dst, &h, sizeof(h), cudaMemcpyHostToDevice));
  MGPU_CUDA(cudaMemset(dbar, 0, sizeof(unsigned long long)));
  MGPU_CUDA(cudaMemset(drec, 0, sizeof(MgpuIterRec)));
  KrylovArgs a{};
  a.n = n;
  a.row_ptr = drp;
  a.col = dcol;
  a.diag = ddiag;
  a.aval = dval;
  a.fval = dfval;
  a.b = db;
  a.x = dx;
  a.r = dkw;
  a.r0 = dkw + n;
  a.p = dkw + 2l * n;
  a.v = dkw + 3l * n;
  a.s = dkw + 4l * n;
  a.t = dkw + 5l * n;
  a.ph = dkw + 6l * n;
  a.sh = dkw + 7l * n;
  a.z = dkw + 8l * n;
  a.w = dkw + 9l * n;
  a.nlev_lo = P.nlo;
  a.lo_ptr = dlop;
  a.lo_rows = dlor;
  a.nlev_up = P.nup;
  a.up_ptr = dupp;
  a.up_rows = dupr;
  a.lt_pos = dmir;
  a.tol = tol;
  a.maxit = maxit;
  a.precond = precond;
  a.zero_x = 0;
  a.mpi_mode = norm_mode ? 1 : 0;
  a.partials = dpart;
  a.bar = dbar;
  a.st = dst;
  a.recs = drec;
  a.slot = 0;
  a.ier_breakdown = 0;
  a.ferr = dferr;
  cudaStream_t s = 0;
  if (precond != 1) TRY(launch_factor(a, precond, s));
  if (bicg)
    TRY(launch_krylov_bicgstab(a, s));
  else
    TRY(launch_krylov_pcg(a, s));
  MGPU_CUDA(cudaDeviceSynchronize());
  MgpuIterRec r{};
  MGPU_CUDA(cudaMemcpy(&r, drec, sizeof(r), cudaMemcpyDeviceToHost));
  MGPU_CUDA(cudaMemcpy(&h, dst, sizeof(h), cudaMemcpyDeviceToHost));
  MGPU_CUDA(cudaMemcpy(x, dx, sizeof(double) * n, cudaMemcpyDeviceToHost));
  if (h.timeout) {
    set_error("a bounded device wait ran out (grid barrier)");
    return MGPU_E_TIMEOUT;
  }
  *it = r.lin_it[0];
  *res = r.lin_res[0];
  *ierr = r.lin_ierr[0];
  return 0;
}

int mgpu_pcg_poly_solve(int n, const int32_t* row_ptr, const int32_t* col_idx, const double* val, const double* b,
                        double* x, double tol, int maxit, int precision, int cheb_degree, int* it, double* res,
                        int* ierr) {
  if (n <= 0 || !row_ptr || !col_idx || !val || !b || !x || !it || !res || !ierr || maxit < 0 ||
      (precision != MGPU_PREC_MIXED && precision != MGPU_PREC_FP64_POLY) || n > kMixedMaxRows) {
    set_error("mgpu_pcg_poly_solve: invalid argument");
    return MGPU_E_ARG;
  }
  Pattern P;
  analyse(n, row_ptr, col_idx, P);
  *it = 0;
  *res = 0.0;
  *ierr = 0;
  if (!P.full_diag) {
    set_error("mgpu_pcg_poly_solve: a row has no diagonal entry");
    return MGPU_E_ARG;
  }
  int k = cheb_degree;
  double ratio = g_cheb_ratio;
  if (k <= 0) cheb_params(n, k, ratio);  // the tuning keys, as a case's pressure solve of n rows
  return precision == MGPU_PREC_MIXED ? poly_solve<float>(n, P, val, b, x, tol, maxit, k, ratio, it, res, ierr)
                                      : poly_solve<double>(n, P, val, b, x, tol, maxit, k, ratio, it, res, ierr);
}

int mgpu_csr_matvec(int n, const int32_t* row_ptr, const int32_t* col_idx, const double* val, const double* x,
                    double* y) {
  if (n <= 0 || !row_ptr || !col_idx || !val || !x || !y) {
    set_error("mgpu_csr_matvec: invalid argument");
    return MGPU_E_ARG;
  }
  std::vector<int> rp(n + 1);
  for (int i = 0; i <= n; ++i) rp[i] = row_ptr[i] - 1;
  const int nnz = rp[n];
  std::vector<int> col(nnz);
  for (int k = 0; k < nnz; ++k) col[k] = col_idx[k] - 1;
  DevBuf B;
  int *drp, *dcol;
  double *dval, *dx, *dy;
  TRY(B.up(drp, rp.data(), n + 1));
  TRY(B.up(dcol, col.data(), nnz));
  TRY(B.up(dval, val, nnz));
  TRY(B.up(dx, x, n));
  TRY(B.alloc(dy, n));
  TRY(launch_spmv(n, drp, dcol, dval, dx, dy, 0));
  MGPU_CUDA(cudaMemcpy(y, dy, sizeof(double) * n, cudaMemcpyDeviceToHost));
  return 0;
}

int mgpu_build_connectivity(const MgpuMesh* mesh, int32_t* cf_ptr, int32_t* cf, int32_t* c2c_ptr, int32_t* c2c,
                            int32_t* row_ptr, int32_t* col_idx, int32_t* nnz) {
  HostMesh m;
  std::string why;
  if (int e = load_host_mesh(mesh, m, why)) {
    set_error(why);
    return e;
  }
  HostTopo t;
  build_topology(m, t);
  for (int i = 0; i <= m.N; ++i) {
    cf_ptr[i] = t.cf_ptr[i] + 1;
    c2c_ptr[i] = t.c2c_ptr[i] + 1;
    row_ptr[i] = t.row_ptr[i] + 1;
  }
  for (size_t k = 0; k < t.cf.size(); ++k) cf[k] = t.cf[k] + 1;
  for (size_t k = 0; k < t.c2c.size(); ++k) c2c[k] = t.c2c[k] + 1;
  for (size_t k = 0; k < t.col.size(); ++k) col_idx[k] = t.col[k] + 1;
  *nnz = (int32_t)t.col.size();
  return 0;
}

int mgpu_geometry(const MgpuMesh* mesh, double* xf, double* sf, double* area, double* vol, double* xc,
                  double* lf) {
  HostMesh m;
  std::string why;
  if (int e = load_host_mesh(mesh, m, why)) {
    set_error(why);
    return e;
  }
  HostTopo t;
  build_topology(m, t);
  DevBuf B;
  DeviceCase d{};
  d.N = m.N;
  d.F = m.F;
  const long N = m.N, F = m.F;
  double *x, *pcen;
  int *fptr, *fnodes;
  TRY(B.up(d.c0, m.c0.data(), F));
  TRY(B.up(d.c1, m.c1.data(), F));
  TRY(B.up(d.cf_ptr, t.cf_ptr.data(), N + 1));
  TRY(B.up(d.cf, t.cf.data(), t.cf.size()));
  TRY(B.up(x, m.x.data(), m.x.size()));
  TRY(B.up(fptr, m.fptr.data(), m.fptr.size()));
  TRY(B.up(fnodes, m.fnodes.data(), m.fnodes.size()));
  TRY(B.alloc(pcen, 3 * N));
  TRY(B.alloc(d.xf, 3 * F));
  TRY(B.alloc(d.sf, 3 * F));
  TRY(B.alloc(d.area, F));
  TRY(B.alloc(d.lf, F));
  TRY(B.alloc(d.vol, N));
  TRY(B.alloc(d.xc, 3 * N));
  TRY(B.alloc(d.dn, F));
  TRY(B.alloc(d.dsf, F));
  TRY(B.alloc(d.Dm, F));
  TRY(B.alloc(d.tv, 3 * F));
  TRY(B.alloc(d.mnc, F));
  AsmParams P{};
  P.mu = 1.0;
  P.nonorth_corr = 1.0;
  TRY(geometry_setup(d, x, fptr, fnodes, pcen, P, 0));
  MGPU_CUDA(cudaDeviceSynchronize());
  auto down3 = [&](double* dst, const double* src, long n) -> int {
    std::vector<double> h(3 * n);
    MGPU_CUDA(cudaMemcpy(h.data(), src, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost));
    for (long i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) dst[3 * i + k] = h[k * n + i];
    return 0;
  };
  TRY(down3(xf, d.xf, F));
  TRY(down3(sf, d.sf, F));
  TRY(down3(xc, d.xc, N));
  MGPU_CUDA(cudaMemcpy(area, d.area, sizeof(double) * F, cudaMemcpyDeviceToHost));
  MGPU_CUDA(cudaMemcpy(vol, d.vol, sizeof(double) * N, cudaMemcpyDeviceToHost));
  MGPU_CUDA(cudaMemcpy(lf, d.lf, sizeof(double) * F, cudaMemcpyDeviceToHost));
  return 0;
}

int mgpu_rcm_order(const MgpuMesh* mesh, int32_t* new_of_old) {
  HostMesh m;
  std::string why;
  if (!new_of_old) return MGPU_E_ARG;
  if (int e = load_host_mesh(mesh, m, why)) {
    set_error(why);
    return e;
  }
  std::vector<int> o;
  rcm_order(m, o);
  std::copy(o.begin(), o.end(), new_of_old);
  return 0;
}

}  // extern "C"
