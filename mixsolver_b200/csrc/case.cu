// case.cu -- the C-ABI of include/mixgpu.h: case lifetime, field transfer,
// the SIMPLE and PISO drivers, and the stand-alone entry points.
//
// A case keeps mesh, geometry, matrices, fields and Krylov work resident in
// HBM from mgpu_case_create to mgpu_case_destroy. A run enqueues every outer
// iteration on the case's stream without host round trips: kernels return at
// once after an abort (breakdown, non-finite value, convergence), so the
// reference's early returns hold while the host only syncs at the end.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "assembly.cuh"
#include "case.cuh"
#include "case_host.h"
#include "device_topo.h"
#include "mesh_host.h"

namespace mgpu {

static thread_local std::string g_err;
static int g_device = 0;
static std::mutex g_stream_mu;
static std::map<int, std::vector<cudaStream_t>> g_streams;

void set_error(const std::string& msg) { g_err = msg; }

cudaStream_t acquire_stream() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  {
    std::lock_guard<std::mutex> lk(g_stream_mu);
    auto& v = g_streams[dev];
    if (!v.empty()) {
      cudaStream_t s = v.back();
      v.pop_back();
      return s;
    }
  }
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  return s;
}

void release_stream(cudaStream_t s) {
  if (!s) return;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_stream_mu);
  g_streams[dev].push_back(s);
}

// Make sure at least n streams wait in the pool of the current device.
int prewarm_streams(int n) {
  int dev = 0;
  MGPU_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_stream_mu);
  auto& v = g_streams[dev];
  while ((int)v.size() < n) {
    cudaStream_t s = nullptr;
    MGPU_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    v.push_back(s);
  }
  return 0;
}

int copy_sync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
  if (bytes == 0) return 0;
  MGPU_CUDA(cudaMemcpyAsync(dst, src, bytes, kind, s));
  MGPU_CUDA(cudaStreamSynchronize(s));
  return 0;
}

__global__ void k_planes_to_cells(const double* __restrict__ src, long n, int planes, bool grad,
                                  double* __restrict__ dst) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;  // output index: cell-major
  if (t >= n * planes) return;
  const long i = t / planes;
  const int k = (int)(t - i * planes);
  const int q = grad ? (k % 3) * 3 + k / 3 : k;
  dst[t] = src[q * n + i];
}

__global__ void k_cells_to_planes(const double* __restrict__ src, long n, int planes, double* __restrict__ dst) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;  // output index: plane-major
  if (t >= n * planes) return;
  const long k = t / n;
  const long i = t - k * n;
  dst[t] = src[planes * i + k];
}

// iface_vel(:, f) / iface_p(f) of the listed faces (0-based), u AoS (3, n)
// cf_first: 1 for a cell-face entry whose CSR slot no earlier entry of the
// same cell has (boundary faces, which have no slot: 0)
__global__ void k_slot_first(int N, const int* __restrict__ cf_ptr, const int* __restrict__ cf_slot,
                             unsigned char* __restrict__ first) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int kb = cf_ptr[c], ke = cf_ptr[c + 1];
  for (int k = kb; k < ke; ++k) {
    const int s = cf_slot[k];
    bool f = s >= 0;
    for (int j = kb; j < k && f; ++j) f = cf_slot[j] != s;
    first[k] = f ? 1 : 0;
  }
}

__global__ void k_iface_scatter(int n, const int* __restrict__ faces, const double* __restrict__ u,
                                const double* __restrict__ p, long F, double* ivel, double* ip) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int f = faces[k];
  if (u) {
    ivel[f] = u[3l * k];
    ivel[F + f] = u[3l * k + 1];
    ivel[2 * F + f] = u[3l * k + 2];
  }
  if (p) ip[f] = p[k];
}

// iface_T(f) / iface_q(f) / iface_T_mode(f) of the listed faces (0-based)
__global__ void k_iface_scatter_T(int n, const int* __restrict__ faces, const double* __restrict__ T,
                                  const double* __restrict__ q, const int* __restrict__ mode, double* iT, double* iq,
                                  int* itm) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int f = faces[k];
  if (T) iT[f] = T[k];
  if (q) iq[f] = q[k];
  if (mode) itm[f] = mode[k];
}

// the owner cell's u (AoS), p and T of every interface face
__global__ void k_iface_gather(int n, const int* __restrict__ faces, const int* __restrict__ c0,
                               const double* __restrict__ u, const double* __restrict__ p,
                               const double* __restrict__ T, long N, double* out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = c0[faces[k]];
  out[5l * k] = u[c];
  out[5l * k + 1] = u[N + c];
  out[5l * k + 2] = u[2 * N + c];
  out[5l * k + 3] = p[c];
  out[5l * k + 4] = T[c];
}

int launch_planes_to_cells(const double* src, long n, int planes, bool grad, double* dst, cudaStream_t s) {
  const long tot = n * planes;
  if (tot == 0) return 0;
  k_planes_to_cells<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(src, n, planes, grad, dst);
  MGPU_CUDA(cudaGetLastError());
  return 0;
}

int launch_cells_to_planes(const double* src, long n, int planes, double* dst, cudaStream_t s) {
  const long tot = n * planes;
  if (tot == 0) return 0;
  k_cells_to_planes<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(src, n, planes, dst);
  MGPU_CUDA(cudaGetLastError());
  return 0;
}

int cuda_fail(cudaError_t e, const char* what, const char* file, int line) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e) + " (" + file + ":" + std::to_string(line) + ")";
  return MGPU_E_CUDA;
}

}  // namespace mgpu

using namespace mgpu;

namespace mgpu {
int ensure_stage(MgpuCase* c, size_t n) {
  if (c->stage_n >= n) return 0;
  if (c->stage) MGPU_CUDA(cudaFreeAsync(c->stage, c->stream));
  c->stage = nullptr;
  c->stage_n = 0;
  void* q = nullptr;
  MGPU_CUDA(cudaMallocAsync(&q, sizeof(double) * std::max<size_t>(n, 1), c->stream));
  c->stage = (double*)q;
  c->stage_n = n;
  return 0;
}
}  // namespace mgpu

namespace mgpu {

KrylovArgs base_args(MgpuCase* c) {
  DeviceCase& d = c->d;
  KrylovArgs a{};
  a.n = d.N;
  a.row_ptr = d.row_ptr;
  a.col = d.col;
  a.diag = d.diag;
  a.fval = d.fval;
  const long N = d.N;
  a.r = d.kw;
  a.r0 = d.kw + N;
  a.p = d.kw + 2 * N;
  a.v = d.kw + 3 * N;
  a.s = d.kw + 4 * N;
  a.t = d.kw + 5 * N;
  a.ph = d.kw + 6 * N;
  a.sh = d.kw + 7 * N;
  a.z = d.kw + 8 * N;
  a.w = d.kw + 9 * N;
  a.nlev_lo = d.nlev_lo;
  a.lo_ptr = d.lo_ptr;
  a.lo_rows = d.lo_rows;
  a.nlev_up = d.nlev_up;
  a.up_ptr = d.up_ptr;
  a.up_rows = d.up_rows;
  a.lt_pos = d.lt_pos;
  a.partials = d.partials;
  a.bar = d.bar;
  a.st = d.st;
  a.recs = d.recs;
  a.ferr = d.ferr;
  a.tol = c->ctrl.lin_tol;
  a.maxit = c->ctrl.lin_max;
  return a;
}

cudaEvent_t next_event(MgpuCase* c) {
  if (c->ev_used >= c->ev_pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    c->ev_pool.push_back(e);
  }
  return c->ev_pool[c->ev_used++];
}

MixedArgs mixed_args(const MgpuCase* c, bool bicg) {
  // a system larger than the L2 share given by l2_prefetch_mb streams from
  // DRAM: its SpMV tiles prefetch the next tile's ELL entries
  const bool big = (double)c->d.N * mixed_row_bytes(c->d.ell_w) > g_prefetch_mb * 1048576.0;
  int k = 1;
  double ratio = g_cheb_ratio;
  if (!bicg) cheb_params(c->d.N, k, ratio);
  return MixedArgs{c->d.a32,   c->d.dinv32, c->d.w32,  c->ctrl.mixed_tol > 0.0 ? c->ctrl.mixed_tol : 1e-4,
                   k,          ratio,       c->d.ell_w, c->d.ell_col, c->d.ell_val,
                   c->d.red32, (c->d.ell_col && big) ? 1 : 0, 0.0, c->d.ell_ld, 0,
                   c->d.ell_val64};
}

// The same solves in FP64 throughout (MGPU_PREC_FP64_POLY): PCG keeps one
// Krylov stream and checks b - A x when the recursive residual converges
// (restarting from it when the check fails); BiCGStab solves to the tolerance
// in one pass.
MixedArgsT<double> poly64_args(const MgpuCase* c, bool bicg) {
  const bool big = (double)c->d.N * (16.0 * c->d.ell_w + 8.0 * 10) > g_prefetch_mb * 1048576.0;
  int k = 1;
  double ratio = g_cheb_ratio;
  if (!bicg) cheb_params(c->d.N, k, ratio);
  return MixedArgsT<double>{c->d.a64, c->d.dinv64, c->d.w64, 0.0, k, ratio,
                            c->d.ell_w, c->d.ell_col, c->d.ell_val64, c->d.red32,
                            (c->d.ell_col && big) ? 1 : 0, 0.0, c->d.ell_ld};
}

// factor (if needed) + solve; precond 0 ILU0, 1 Jacobi, 2 IC0. The mixed form
// (ctrl.precision) runs FP32-inner / FP64-refinement solves with Jacobi or
// Chebyshev-Jacobi; the FP64 polynomial form the same solvers in FP64.
int krylov(MgpuCase* c, KrylovArgs a, bool bicg, cudaStream_t s) {
  if (c->ctrl.precision == MGPU_PREC_MIXED || c->ctrl.precision == MGPU_PREC_FP64_POLY) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->profiling) {
      e0 = next_event(c);
      e1 = next_event(c);
      cudaEventRecord(e0, s);
    }
    a.precond = 1;
    if (c->ctrl.precision == MGPU_PREC_MIXED) {
      const MixedArgs m = mixed_args(c, bicg);
      TRY(bicg ? launch_bicgstab_mixed(a, m, s) : launch_pcg_mixed(a, m, s));
    } else {
      const MixedArgsT<double> m = poly64_args(c, bicg);
      TRY(bicg ? launch_bicgstab_poly64(a, m, s) : launch_pcg_poly64(a, m, s));
    }
    c->launches++;
    if (c->profiling) cudaEventRecord(e1, s);
    return 0;
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (c->profiling) {
    e0 = next_event(c);
    e1 = next_event(c);
    cudaEventRecord(e0, s);
  }
  if (a.precond != 1) {
    TRY(launch_factor(a, a.precond, s));
    c->launches++;
  }
  if (bicg)
    TRY(launch_krylov_bicgstab(a, s));
  else
    TRY(launch_krylov_pcg(a, s));
  c->launches++;
  if (c->profiling) cudaEventRecord(e1, s);
  return 0;
}

KrylovArgs mom_args(MgpuCase* c, int comp, bool transient) {
  KrylovArgs a = base_args(c);
  a.aval = c->d.aval;
  a.b = c->d.rhs;
  a.x = c->d.u + (long)comp * c->d.N;
  a.precond = c->ctrl.mom_solver == MGPU_MOM_JACOBI ? 1 : 0;
  a.zero_x = 0;
  a.mpi_mode = transient ? 1 : 0;
  a.slot = comp;
  a.ier_breakdown = c->P.pimple ? 53 : (transient ? 33 : 20);
  return a;
}

KrylovArgs ppe_args(MgpuCase* c, int slot, bool transient) {
  KrylovArgs a = base_args(c);
  a.aval = c->d.pval;
  a.b = c->d.rhs;
  a.x = c->d.pp;
  a.precond = c->ctrl.ppe_precond == MGPU_PPE_IC0 ? 2 : (c->ctrl.ppe_precond == MGPU_PPE_ILU0 ? 0 : 1);
  a.zero_x = 1;
  a.mpi_mode = transient ? 1 : 0;
  a.slot = slot;
  a.ier_breakdown = c->P.pimple ? 54 : (transient ? 34 : 21);
  return a;
}

KrylovArgs temperature_args(MgpuCase* c, int slot, bool transient) {
  KrylovArgs a = base_args(c);
  a.aval = c->d.aval;
  a.b = c->d.rhs;
  a.x = c->d.T;
  a.precond = c->ctrl.mom_solver == MGPU_MOM_JACOBI ? 1 : 0;
  a.zero_x = 0;
  a.mpi_mode = transient ? 1 : 0;
  a.slot = slot;
  a.ier_breakdown = c->P.pimple ? 55 : (transient ? 35 : 22);
  return a;
}

namespace {

// The temperature equation of a driver step (mod_uns_simple.f90:200-210,
// mod_uns_simple_mpi.f90:467-479 / 750-760): T before the solve kept for
// dT_max, the assembly (limiter first with conv_blend), the solve from the
// current T with the momentum solver into record slot `slot`.
int temperature_step(MgpuCase* c, int slot, bool transient) {
  DeviceCase& d = c->d;
  cudaStream_t s = c->stream;
  MGPU_CUDA(cudaMemcpyAsync(d.Tprev, d.T, sizeof(double) * d.N, cudaMemcpyDeviceToDevice, s));
  TRY(launch_temperature(d, c->P, s));
  c->launches += c->P.conv_blend > 0.0 ? 2 : 1;
  return krylov(c, temperature_args(c, slot, transient), true, s);  // slots past the record: not logged
}

int momentum_solve(MgpuCase* c, int comp, bool transient) {
  return krylov(c, mom_args(c, comp, transient), true, c->stream);
}

int ppe_solve(MgpuCase* c, int slot, bool transient) { return krylov(c, ppe_args(c, slot, transient), false, c->stream); }

// The momentum predictor: per component the assembly, then its solve. With
// conv_blend = 0 the interior faces of all three components are assembled in
// one pass and each component then adds its boundary faces, sources and
// relaxation right before its solve (the boundary values use the components
// solved before it, as in the reference's loop); with the limited convection
// scheme every component is assembled whole after the previous solve.
int assemble_and_solve_momentum(MgpuCase* c, bool transient) {
  DeviceCase& d = c->d;
  const AsmParams& P = c->P;
  cudaStream_t s = c->stream;
  const bool fused = !(P.conv_blend > 0.0);
  if (fused) {
    TRY(launch_mom_interior(d, P, s));
    c->launches++;
  }
  for (int comp = 0; comp < 3; ++comp) {
    if (fused) {
      TRY(launch_mom_finish(d, P, comp, s));
    } else {
      TRY(launch_limiter(d, P, comp, s));
      c->launches++;
      TRY(launch_momentum(d, P, comp, s));
    }
    c->launches++;
    TRY(momentum_solve(c, comp, transient));
  }
  return 0;
}

}  // namespace

int reset_status(MgpuCase* c, int ts_order, int nrec) {
  DevStatus h{};
  h.ts_order = ts_order;
  h.nan_key = ~0ull;
  h.it_limit = nrec > 1 ? nrec - 1 : 0;
  h.spin_limit = g_spin_limit;
  h.poll_ns = g_poll_ns;
  MGPU_CUDA(cudaMemcpyAsync(c->d.st, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  MGPU_CUDA(cudaMemsetAsync(c->d.bar, 0, sizeof(unsigned long long), c->stream));
  MGPU_CUDA(cudaMemsetAsync(c->d.recs, 0, sizeof(MgpuIterRec) * (size_t)nrec, c->stream));
  return 0;
}

int ensure_recs(MgpuCase* c, int n) {
  if (n <= c->d.rec_cap) return 0;
  MgpuIterRec* r = nullptr;
  TRY(c->alloc(r, (size_t)n));
  c->d.recs = r;  // the old buffer stays owned by the case until destroy
  c->d.rec_cap = n;
  return 0;
}

namespace {

int begin_run(MgpuCase* c) {
  c->P.pimple = 0;  // mgpu_pimple_run sets it after this
  c->ev_used = 0;
  c->launches = 0;
  c->timing = MgpuTiming{};
  if (!c->ev_run0) {
    MGPU_CUDA(cudaEventCreate(&c->ev_run0));
    MGPU_CUDA(cudaEventCreate(&c->ev_run1));
  }
  MGPU_CUDA(cudaEventRecord(c->ev_run0, c->stream));
  return 0;
}

int end_run(MgpuCase* c, int nsteps_done, MgpuIterRec* log, int logcap, int* nrec, int* ier) {
  MGPU_CUDA(cudaEventRecord(c->ev_run1, c->stream));
  DevStatus h{};
  MGPU_CUDA(cudaMemcpyAsync(&h, c->d.st, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  MGPU_CUDA(cudaStreamSynchronize(c->stream));
  (void)nsteps_done;
  const int done = h.cur_it;
  if (nrec) *nrec = done;
  if (log && logcap > 0 && done > 0)
    TRY(copy_sync(log, c->d.recs, sizeof(MgpuIterRec) * (size_t)std::min(done, logcap),
                         cudaMemcpyDeviceToHost, c->stream));
  if (ier) *ier = h.ier;
  float ms = 0.f;
  cudaEventElapsedTime(&ms, c->ev_run0, c->ev_run1);
  c->timing.total_ms = ms;
  c->timing.gpu_launches = c->launches;
  if (c->profiling) {
    double kms = 0.0;
    for (size_t i = 0; i + 1 < c->ev_used; i += 2) {
      float t = 0.f;
      cudaEventElapsedTime(&t, c->ev_pool[i], c->ev_pool[i + 1]);
      kms += t;
    }
    c->timing.krylov_launches = (int64_t)(c->ev_used / 2);
    c->timing.krylov_ms = kms;
  }
  if (h.timeout) {
    set_error("a bounded device wait ran out (grid barrier)");
    return MGPU_E_TIMEOUT;
  }
  return 0;
}

// The armed last iteration of mgpu_simple_run_fields: gp and gu transposed to
// cell-major order into stage2 on the case's stream, then gp, gu and apc
// copied to the caller's page-locked arrays on copy_stream, which runs beside
// the rest of the iteration (nothing later in the run writes these fields).
int enqueue_early_copy(MgpuCase* c) {
  const long N = c->d.N;
  cudaStream_t s = c->stream;
  MgpuCase::EarlyCopy& e = c->early;
  if (e.gp) TRY(launch_planes_to_cells(c->d.gp, N, 3, false, c->stage2, s));
  if (e.gu) TRY(launch_planes_to_cells(c->d.gu, N, 9, true, c->stage2 + 3 * N, s));
  c->launches += (e.gp ? 1 : 0) + (e.gu ? 1 : 0);
  MGPU_CUDA(cudaEventRecord(c->ev_early, s));
  MGPU_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev_early, 0));
  cudaStream_t cs = c->copy_stream;
  if (e.gp) MGPU_CUDA(cudaMemcpyAsync(e.gp, c->stage2, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, cs));
  if (e.gu) MGPU_CUDA(cudaMemcpyAsync(e.gu, c->stage2 + 3 * N, sizeof(double) * 9 * N, cudaMemcpyDeviceToHost, cs));
  if (e.apc) MGPU_CUDA(cudaMemcpyAsync(e.apc, c->d.apc, sizeof(double) * N, cudaMemcpyDeviceToHost, cs));
  MGPU_CUDA(cudaEventRecord(c->ev_copied, cs));
  e.armed = false;
  e.done = true;
  return 0;
}

int outer_iteration(MgpuCase* c, bool transient) {
  DeviceCase& d = c->d;
  const AsmParams& P = c->P;
  cudaStream_t s = c->stream;
  TRY(launch_begin_iter(d, transient ? 1 : 0, c->ctrl.time_scheme, P.inlet_ramp, s));
  c->launches++;
  TRY(assemble_and_solve_momentum(c, transient));
  TRY(launch_apc(d, transient ? 1.0 : P.alpha_u, s));
  TRY(launch_gradients(d, P, s));
  if (c->early.armed) TRY(enqueue_early_copy(c));
  TRY(launch_rhiechow(d, P, s));
  c->launches += 3;
  if (c->has_outflow) {
    TRY(launch_outflow(d, s));
    c->launches++;
  }
  const int ncorr = transient ? std::max(1, c->ctrl.n_correct) : 1;
  for (int icorr = 0; icorr < ncorr; ++icorr) {
    TRY(launch_ppe(d, P, s));
    c->launches++;
    TRY(ppe_solve(c, std::min(3 + icorr, MGPU_MAXSOLVE - 1), transient));
    TRY(launch_correct(d, P, s));
    c->launches += 2;
  }
  if (d.energy) TRY(temperature_step(c, 3 + ncorr, transient));
  TRY(launch_diag(d, P, transient ? 1 : 0, s));
  c->launches += 2;
  return 0;
}

// One PIMPLE time step (pimple_run_mpi at one rank, mod_uns_simple_mpi.f90:
// 676-760): the history shift once, then n_outer_iter outer iterations of the
// relaxed momentum predictor (P.pimple), apc = ap / alpha_u, gradients,
// Rhie-Chow fluxes, outflow rescale and n_correct pressure corrections; the
// step's diagnostics at the end.
int pimple_step(MgpuCase* c) {
  DeviceCase& d = c->d;
  const AsmParams& P = c->P;
  cudaStream_t s = c->stream;
  TRY(launch_begin_iter(d, 1, c->ctrl.time_scheme, P.inlet_ramp, s));
  c->launches++;
  const int n_outer = std::max(1, c->ctrl.n_outer_iter);
  const int ncorr = std::max(1, c->ctrl.n_correct);
  for (int io = 0; io < n_outer; ++io) {
    TRY(assemble_and_solve_momentum(c, true));
    TRY(launch_apc(d, P.alpha_u, s));
    TRY(launch_gradients(d, P, s));
    TRY(launch_rhiechow(d, P, s));
    c->launches += 3;
    if (c->has_outflow) {
      TRY(launch_outflow(d, s));
      c->launches++;
    }
    for (int icorr = 0; icorr < ncorr; ++icorr) {
      TRY(launch_ppe(d, P, s));
      c->launches++;
      TRY(ppe_solve(c, std::min(3 + icorr, MGPU_MAXSOLVE - 1), true));
      TRY(launch_correct(d, P, s));
      c->launches += 2;
    }
    if (io + 1 < n_outer) {
      TRY(launch_outer_accum(d, s));
      c->launches++;
    }
  }
  // the temperature once per step, with the final corrected velocity
  if (d.energy) TRY(temperature_step(c, 3 + ncorr, true));
  TRY(launch_diag(d, P, 1, s));
  c->launches += 2;
  return 0;
}

}  // namespace
}  // namespace mgpu

extern "C" {

int mgpu_version(void) { return 100; }

const char* mgpu_last_error(void) { return g_err.c_str(); }

int mgpu_set_device(int device) {
  MGPU_CUDA(cudaSetDevice(device));
  g_device = device;
  return 0;
}

int mgpu_case_create(const MgpuMesh* mesh, const MgpuCtrl* ctrl, MgpuCase** out, int* ier) {
  if (ier) *ier = 0;
  if (!out || !ctrl) {
    set_error("mgpu_case_create: null argument");
    return MGPU_E_ARG;
  }
  *out = nullptr;
  HostMesh hm;
  std::string why;
  if (int e = load_host_mesh(mesh, hm, why)) {
    set_error(why);
    return e;
  }
  std::vector<DevGroup> groups;
  std::vector<int> fgrp;
  int bier = 0;
  if (int e = build_groups(hm, *ctrl, groups, fgrp, bier, why)) {
    if (ier) *ier = bier;
    set_error(why);
    return e;
  }
  if (ctrl->conv_blend < 0.0 || ctrl->alpha_u <= 0.0 || ctrl->lin_max < 0) {
    set_error("ctrl: invalid alpha_u / conv_blend / lin_max");
    return MGPU_E_ARG;
  }
  const bool poly = ctrl->precision == MGPU_PREC_MIXED || ctrl->precision == MGPU_PREC_FP64_POLY;
  if (ctrl->precision < MGPU_PREC_FP64 || ctrl->precision > MGPU_PREC_FP64_POLY) {
    set_error("mgpu_case_create: unknown precision");
    return MGPU_E_ARG;
  }
  if (poly && hm.N > kMixedMaxRows) {
    set_error("mgpu_case_create: the mixed-precision and FP64 polynomial forms take at most 2^23 cells");
    return MGPU_E_ARG;
  }
  MGPU_CUDA(cudaSetDevice(g_device));
  MgpuCase* c = new MgpuCase();
  auto fail = [&](int e) {
    delete c;
    return e;
  };
  c->ctrl = *ctrl;
  c->stream = acquire_stream();
  if (!c->stream) {
    set_error("cudaStreamCreate failed");
    return fail(MGPU_E_CUDA);
  }
  DeviceCase& d = c->d;
  d.N = hm.N;
  d.F = hm.F;
  const long N = d.N, F = d.F;
  int e = 0;
  double *x = nullptr, *pcen = nullptr;
  int *fptr = nullptr, *fnodes = nullptr;
  if ((e = c->upload(d.c0, hm.c0)) || (e = c->upload(d.c1, hm.c1)) || (e = c->upload(d.fgrp, fgrp)) ||
      (e = c->upload(d.groups, groups)))
    return fail(e);
  // the integer mesh pipeline on the device (build_connectivity, build_cell_csr,
  // slot maps, level sets): device_topo.cu
  const TopoAlloc keep = [c](int*& p, size_t n) { return c->alloc(p, n); };
  {
    DeviceTopo t;
    // the mixed and FP64 polynomial forms run no triangular sweeps
    const bool levels = ctrl->precision == MGPU_PREC_FP64;
    if ((e = device_topology(d.N, d.F, d.c0, d.c1, t, keep, c->stream, levels))) return fail(e);
    d.cf_ptr = t.cf_ptr;
    d.cf = t.cf;
    d.cf_slot = t.cf_slot;
    d.row_ptr = t.row_ptr;
    d.col = t.col;
    d.diag = t.diag;
    d.lt_pos = t.mirror;
    d.lo_ptr = t.lo_ptr;
    d.lo_rows = t.lo_rows;
    d.up_ptr = t.up_ptr;
    d.up_rows = t.up_rows;
    d.nlev_lo = t.nlev_lo;
    d.nlev_up = t.nlev_up;
    d.nnz = t.nnz;
    if ((e = c->alloc(d.cf_first, (size_t)t.ncf))) return fail(e);
    k_slot_first<<<ceil_div(N, 256), 256, 0, c->stream>>>(d.N, d.cf_ptr, d.cf_slot, d.cf_first);
    MGPU_CUDA(cudaGetLastError());
  }
  d.ngroups = (int)groups.size();
  if ((e = c->alloc(d.xf, 3 * F)) || (e = c->alloc(d.sf, 3 * F)) || (e = c->alloc(d.area, F)) ||
      (e = c->alloc(d.lf, F)) || (e = c->alloc(d.vol, N)) || (e = c->alloc(d.xc, 3 * N)) ||
      (e = c->alloc(d.dn, F)) || (e = c->alloc(d.dsf, F)) || (e = c->alloc(d.Dm, F)) ||
      (e = c->alloc(d.tv, 3 * F)) || (e = c->alloc(d.mnc, F)) || (e = c->alloc(d.u, 3 * N)) ||
      (e = c->alloc(d.p, N)) || (e = c->alloc(d.gp, 3 * N)) || (e = c->alloc(d.gu, 9 * N)) ||
      (e = c->alloc(d.flux, F)) || (e = c->alloc(d.apc, N)) || (e = c->alloc(d.ap, N)) ||
      (e = c->alloc(d.rhs, N)) || (e = c->alloc(d.pp, N)) || (e = c->alloc(d.uo, 3 * N)) ||
      (e = c->alloc(d.u_old, 3 * N)) || (e = c->alloc(d.u_old_old, 3 * N)) || (e = c->alloc(d.psi, N)) ||
      (e = c->alloc(d.af, F)) || (e = c->alloc(d.aval, d.nnz)) || (e = c->alloc(d.pval, d.nnz)) ||
      (e = c->alloc(d.fval, d.nnz)) || (e = c->alloc(d.kw, 10 * N)) ||
      (ctrl->precision == MGPU_PREC_MIXED &&
       ((e = c->alloc(d.a32, d.nnz)) || (e = c->alloc(d.dinv32, N)) || (e = c->alloc(d.w32, 10 * N)))) ||
      (ctrl->precision == MGPU_PREC_FP64_POLY &&
       ((e = c->alloc(d.a64, d.nnz)) || (e = c->alloc(d.dinv64, N)) || (e = c->alloc(d.w64, 10 * N)))) ||
      (poly && (e = c->alloc(d.red32, (size_t)mixed_red_words(N)))) ||
      (e = c->alloc(d.partials, 4 * 4096)) ||
      (e = c->alloc(d.bar, 1)) || (e = c->alloc(d.ferr, 1)) || (e = c->alloc(d.st, 1)) ||
      (e = c->alloc(d.ramp, 2)))
    return fail(e);
  {
    const double one[2] = {1.0, 1.0};  // the ramp factors of a fresh case
    MGPU_CUDA(cudaMemcpyAsync(d.ramp, one, sizeof(one), cudaMemcpyHostToDevice, c->stream));
  }
  if ((e = ensure_recs(c, 64))) return fail(e);
  if (poly) {
    // column-major ELL copy of the pattern for the polynomial forms' SpMV (rows of at most 8 entries)
    int w = 0, *ell = nullptr;
    long ld = 0;
    if ((e = device_ell(d.N, d.row_ptr, d.col, 8, w, ld, ell, keep, c->stream))) return fail(e);
    if (ell) {
      d.ell_col = ell;
      // values zero in the padding rows
      // FP64 values in both forms (the mixed form's conjugate-gradient
      // product, the polynomial form's every product), FP32 in the mixed form
      if ((e = c->alloc(d.ell_val64, (size_t)w * ld))) return fail(e);
      MGPU_CUDA(cudaMemsetAsync(d.ell_val64, 0, sizeof(double) * (size_t)w * ld, c->stream));
      if (ctrl->precision == MGPU_PREC_MIXED) {
        if ((e = c->alloc(d.ell_val, (size_t)w * ld))) return fail(e);
        MGPU_CUDA(cudaMemsetAsync(d.ell_val, 0, sizeof(float) * (size_t)w * ld, c->stream));
      }
      d.ell_w = w;
      d.ell_ld = (int)ld;
    }
  }
  // geometry (device), scratch for the node arrays and provisional centres
  std::vector<int> fptr_h(hm.fptr.begin(), hm.fptr.end());
  if ((e = c->upload(x, hm.x)) || (e = c->upload(fptr, fptr_h)) || (e = c->upload(fnodes, hm.fnodes)) ||
      (e = c->alloc(pcen, 3 * N)))
    return fail(e);
  AsmParams& P = c->P;
  P = AsmParams{};
  P.rho = ctrl->rho;
  P.mu = ctrl->mu;
  P.alpha_u = ctrl->alpha_u;
  P.alpha_p = ctrl->alpha_p;
  P.conv_blend = ctrl->conv_blend;
  P.nonorth_corr = ctrl->nonorth_corr;
  P.dt = ctrl->dt;
  P.outer_tol = ctrl->outer_tol;
  P.inlet_ramp = ctrl->inlet_ramp;
  for (int k = 0; k < 3; ++k) P.body_force[k] = ctrl->body_force[k];
  P.has_body_force = (ctrl->body_force[0] != 0.0 || ctrl->body_force[1] != 0.0 || ctrl->body_force[2] != 0.0);
  P.boussinesq = ctrl->boussinesq ? 1 : 0;
  P.cp = ctrl->cp;
  P.k_cond = ctrl->k_cond;
  P.tref = ctrl->tref;
  P.beta = ctrl->beta;
  for (int k = 0; k < 3; ++k) P.gravity[k] = ctrl->gravity[k];
  d.energy = ctrl->energy ? 1 : 0;
  // T for every case (the NaN scan reads it; zero without the energy
  // equation), its history, gradient and solve scratch when it is solved
  if ((e = c->alloc(d.T, N))) return fail(e);
  MGPU_CUDA(cudaMemsetAsync(d.T, 0, sizeof(double) * N, c->stream));
  if (d.energy) {
    if ((e = c->alloc(d.T_old, N)) || (e = c->alloc(d.T_old_old, N)) || (e = c->alloc(d.gt, 3 * N)) ||
        (e = c->alloc(d.Tprev, N)) || (ctrl->conv_blend > 0.0 && (e = c->alloc(d.psiT, N))))
      return fail(e);
    MGPU_CUDA(cudaMemsetAsync(d.T_old, 0, sizeof(double) * N, c->stream));
    MGPU_CUDA(cudaMemsetAsync(d.T_old_old, 0, sizeof(double) * N, c->stream));
    MGPU_CUDA(cudaMemsetAsync(d.gt, 0, sizeof(double) * 3 * N, c->stream));
  }
  if (P.boussinesq && !d.energy) {
    set_error("mgpu_case_create: boussinesq needs the energy equation (ctrl.energy)");
    return fail(MGPU_E_ARG);
  }
  P.has_pdir = 0;
  for (int k = 0; k < hm.F; ++k)
    if (hm.c1[k] < 0 && (groups[fgrp[k]].btype == MGPU_BC_POUTLET || groups[fgrp[k]].btype == MGPU_BC_FARFIELD))
      P.has_pdir = 1;
  for (int k = 0; k < hm.F; ++k)
    if (hm.c1[k] < 0 && fgrp[k] >= 0 && groups[fgrp[k]].btype == MGPU_BC_INTERFACE) d.n_iface++;
  if (d.n_iface > 0) {  // the peer's interface values, zero until set (mgpu_interface_set)
    // the interface faces, group by group in bc order, each group in face order
    for (int gi = 0; gi < (int)groups.size(); ++gi)
      if (groups[gi].btype == MGPU_BC_INTERFACE)
        for (int k = 0; k < hm.F; ++k)
          if (hm.c1[k] < 0 && fgrp[k] == gi) c->iface_faces.push_back(k);
    if ((e = c->upload(c->d_iface_faces, c->iface_faces))) return fail(e);
    if ((e = c->alloc(d.iface_vel, 3 * F)) || (e = c->alloc(d.iface_p, F)) || (e = c->alloc(d.iface_T, F)) ||
        (e = c->alloc(d.iface_q, F)) || (e = c->alloc(d.iface_tmode, F)))
      return fail(e);
    MGPU_CUDA(cudaMemsetAsync(d.iface_vel, 0, sizeof(double) * 3 * F, c->stream));
    MGPU_CUDA(cudaMemsetAsync(d.iface_p, 0, sizeof(double) * F, c->stream));
    MGPU_CUDA(cudaMemsetAsync(d.iface_T, 0, sizeof(double) * F, c->stream));
    MGPU_CUDA(cudaMemsetAsync(d.iface_q, 0, sizeof(double) * F, c->stream));
    MGPU_CUDA(cudaMemsetAsync(d.iface_tmode, 0, sizeof(int) * F, c->stream));
  }
  for (auto& g : groups)
    if (g.btype == MGPU_BC_OUTFLOW) c->has_outflow = 1;
  P.has_outflow = c->has_outflow;
  // each cell's boundary faces that carry a group, in the order of its face list
  if ((e = device_boundary_lists(d.N, d.cf_ptr, d.cf, d.c1, d.fgrp, d.bf_ptr, d.bf, keep, c->stream)) ||
      (e = c->alloc(d.mom_ap, N)) || (e = c->alloc(d.mom_rhs, 3 * N)))
    return fail(e);
  if (c->has_outflow) {
    // the faces of outflow_mass_sums' two sums, each in face order
    std::vector<int> req, out;
    for (int k = 0; k < hm.F; ++k) {
      if (hm.c1[k] >= 0 || fgrp[k] < 0) continue;
      const int bt = groups[fgrp[k]].btype;
      if (bt == MGPU_BC_OUTFLOW)
        out.push_back(k);
      else if (bt != MGPU_BC_POUTLET && bt != MGPU_BC_FARFIELD)
        req.push_back(k);
    }
    if ((e = c->upload(d.of_req, req)) || (e = c->upload(d.of_out, out))) return fail(e);
    d.n_of_req = (int)req.size();
    d.n_of_out = (int)out.size();
  }
  DeviceCase dd = d;
  DevStatus h0{};
  h0.nan_key = ~0ull;
  MGPU_CUDA(cudaMemcpyAsync(d.st, &h0, sizeof(h0), cudaMemcpyHostToDevice, c->stream));
  if ((e = geometry_setup(dd, x, fptr, fnodes, pcen, P, c->stream))) return fail(e);
  // init_fields: everything at rest, apc = 1
  MGPU_CUDA(cudaMemsetAsync(d.u, 0, sizeof(double) * 3 * N, c->stream));
  MGPU_CUDA(cudaMemsetAsync(d.p, 0, sizeof(double) * N, c->stream));
  MGPU_CUDA(cudaMemsetAsync(d.flux, 0, sizeof(double) * F, c->stream));
  MGPU_CUDA(cudaMemsetAsync(d.u_old, 0, sizeof(double) * 3 * N, c->stream));
  MGPU_CUDA(cudaMemsetAsync(d.u_old_old, 0, sizeof(double) * 3 * N, c->stream));
  MGPU_CUDA(cudaMemsetAsync(d.gp, 0, sizeof(double) * 3 * N, c->stream));
  MGPU_CUDA(cudaMemsetAsync(d.gu, 0, sizeof(double) * 9 * N, c->stream));
  MGPU_CUDA(cudaMemsetAsync(d.af, 0, sizeof(double) * F, c->stream));
  MGPU_CUDA(cudaMemsetAsync(d.bar, 0, sizeof(unsigned long long), c->stream));
  if ((e = launch_fill(d.apc, N, 1.0, c->stream))) return fail(e);
  MGPU_CUDA(cudaStreamSynchronize(c->stream));
  // scalars needing a sequential pass: flux_ref (group/face order) and the
  // smallest vol**(1/3) (CFL estimate); computed once on the host
  std::vector<double> area(F), vol(N);
  TRY(copy_sync(area.data(), d.area, sizeof(double) * F, cudaMemcpyDeviceToHost, c->stream));
  TRY(copy_sync(vol.data(), d.vol, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
  for (long i = 0; i < N; ++i)
    if (!(vol[i] > 0.0)) {
      set_error("mesh: non-positive cell volume");
      return fail(MGPU_E_MESH);
    }
  double uscale = 0.0, area_btot = 0.0;
  for (int gi = 0; gi < (int)groups.size(); ++gi) {
    const DevGroup& g = groups[gi];
    uscale = std::max(std::max(std::max(uscale, norm3(g.lid_vel[0], g.lid_vel[1], g.lid_vel[2])),
                               norm3(g.uvel[0], g.uvel[1], g.uvel[2])),
                      g.uspeed);
    for (int k = 0; k < hm.F; ++k)
      if (fgrp[k] == gi) area_btot = area_btot + area[k];
  }
  if (uscale <= 0.0) uscale = 1.0;
  if (area_btot <= 0.0) area_btot = 1.0;
  P.flux_ref = ctrl->rho * uscale * area_btot;
  double mc = HUGE_VAL;
  for (long i = 0; i < N; ++i) mc = std::min(mc, std::pow(vol[i], 1.0 / 3.0));
  P.min_cbrt_vol = mc;
  *out = c;
  return 0;
}

int mgpu_case_destroy(MgpuCase* c) {
  delete c;
  return 0;
}

int mgpu_case_device_bytes(const MgpuCase* c, int64_t* bytes) {
  if (!c || !bytes) return MGPU_E_ARG;
  *bytes = c->bytes;
  return 0;
}

int mgpu_fields_upload(MgpuCase* c, const double* u, const double* p, const double* flux, const double* u_old,
                       const double* u_old_old) {
  if (!c) return MGPU_E_ARG;
  const long N = c->d.N;
  cudaStream_t s = c->stream;
  // cell-major u(3,N) -> device planes: one copy into the staging buffer, then
  // the transpose on the device (the next copy into the buffer waits for it:
  // same stream)
  auto up3 = [&](double* dst, const double* src) -> int {
    TRY(mgpu::ensure_stage(c, 3 * (size_t)N));
    MGPU_CUDA(cudaMemcpyAsync(c->stage, src, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s));
    TRY(mgpu::launch_cells_to_planes(c->stage, N, 3, dst, s));
    return 0;
  };
  if (u) TRY(up3(c->d.u, u));
  if (u_old) TRY(up3(c->d.u_old, u_old));
  if (u_old_old) TRY(up3(c->d.u_old_old, u_old_old));
  if (p) MGPU_CUDA(cudaMemcpyAsync(c->d.p, p, sizeof(double) * N, cudaMemcpyHostToDevice, s));
  if (flux) MGPU_CUDA(cudaMemcpyAsync(c->d.flux, flux, sizeof(double) * c->d.F, cudaMemcpyHostToDevice, s));
  MGPU_CUDA(cudaStreamSynchronize(s));
  return 0;
}

int mgpu_fields_download(MgpuCase* c, double* u, double* p, double* flux, double* gp, double* gu, double* apc) {
  if (!c) return MGPU_E_ARG;
  const long N = c->d.N;
  cudaStream_t s = c->stream;
  // device planes -> cell-major arrays, transposed on the device into the
  // staging buffer and copied out from there; gu's device plane comp*3+dir
  // goes to the Fortran index comp + 3*dir + 9*cell
  auto down = [&](double* dst, const double* src, int planes, bool grad) -> int {
    TRY(mgpu::ensure_stage(c, (size_t)planes * N));
    TRY(mgpu::launch_planes_to_cells(src, N, planes, grad, c->stage, s));
    MGPU_CUDA(cudaMemcpyAsync(dst, c->stage, sizeof(double) * planes * N, cudaMemcpyDeviceToHost, s));
    return 0;
  };
  if (u) TRY(down(u, c->d.u, 3, false));
  if (gp) TRY(down(gp, c->d.gp, 3, false));
  if (gu) TRY(down(gu, c->d.gu, 9, true));
  if (p) MGPU_CUDA(cudaMemcpyAsync(p, c->d.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  if (apc) MGPU_CUDA(cudaMemcpyAsync(apc, c->d.apc, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  if (flux) MGPU_CUDA(cudaMemcpyAsync(flux, c->d.flux, sizeof(double) * c->d.F, cudaMemcpyDeviceToHost, s));
  MGPU_CUDA(cudaStreamSynchronize(s));
  return 0;
}

static int simple_run_armed(MgpuCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier);

int mgpu_simple_run(MgpuCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier) {
  if (!c || !ier) return MGPU_E_ARG;
  c->early = MgpuCase::EarlyCopy{};
  return simple_run_armed(c, nsteps, log, logcap, nrec, ier);
}

// mgpu_simple_run's body; the early copies of c->early (if any are set) are
// armed for the run's last iteration
static int simple_run_armed(MgpuCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier) {
  if (!c || !ier) return MGPU_E_ARG;
  c->early.armed = false;
  c->early.done = false;
  *ier = 0;
  if (nrec) *nrec = 0;
  int it_max = c->ctrl.outer_max;
  if (nsteps > 0) it_max = std::min(it_max, nsteps);
  if (it_max <= 0) return 0;
  TRY(ensure_recs(c, it_max + 1));
  TRY(begin_run(c));
  TRY(reset_status(c, 0, it_max + 1));
  TRY(launch_fill(c->d.apc, c->d.N, 1.0, c->stream));
  TRY(launch_gradients(c->d, c->P, c->stream));
  c->launches += 2;
  for (int it = 0; it < it_max; ++it) {
    c->early.armed = c->early.gp || c->early.gu || c->early.apc ? it + 1 == it_max : false;
    TRY(outer_iteration(c, false));
    if ((it + 1) % 64 == 0 && it + 1 < it_max) {
      // stop enqueuing once a run has aborted (convergence, breakdown, NaN)
      int ab = 0;
      MGPU_CUDA(cudaMemcpyAsync(&ab, &c->d.st->abort, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      MGPU_CUDA(cudaStreamSynchronize(c->stream));
      if (ab) break;
    }
  }
  return end_run(c, it_max, log, logcap, nrec, ier);
}

namespace {
bool page_locked(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}
}  // namespace

int mgpu_simple_run_fields(MgpuCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier, double* u,
                           double* p, double* flux, double* gp, double* gu, double* apc) {
  if (!c || !ier) return MGPU_E_ARG;
  const bool early = (gp || gu || apc) && (!gp || page_locked(gp)) && (!gu || page_locked(gu)) &&
                     (!apc || page_locked(apc));
  if (early) {
    if (!c->copy_stream) {
      MGPU_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
      MGPU_CUDA(cudaEventCreateWithFlags(&c->ev_early, cudaEventDisableTiming));
      MGPU_CUDA(cudaEventCreateWithFlags(&c->ev_copied, cudaEventDisableTiming));
    }
    const size_t need = 12 * (size_t)c->d.N;
    if (c->stage2_n < need) {
      if (c->stage2) MGPU_CUDA(cudaFreeAsync(c->stage2, c->stream));
      void* q = nullptr;
      MGPU_CUDA(cudaMallocAsync(&q, sizeof(double) * need, c->stream));
      c->stage2 = (double*)q;
      c->stage2_n = need;
    }
  }
  // mgpu_simple_run with the early copies armed for its last iteration
  c->early = MgpuCase::EarlyCopy{};
  if (early) {
    c->early.gp = gp;
    c->early.gu = gu;
    c->early.apc = apc;
  }
  const int rc = simple_run_armed(c, nsteps, log, logcap, nrec, ier);
  const bool done = c->early.done;
  c->early = MgpuCase::EarlyCopy{};
  if (done) MGPU_CUDA(cudaEventSynchronize(c->ev_copied));
  if (rc != 0) return rc;
  // the rest (all of it when the run stopped before its last iteration or the
  // arrays are pageable), as mgpu_fields_download
  return mgpu_fields_download(c, u, p, flux, done ? nullptr : gp, done ? nullptr : gu, done ? nullptr : apc);
}

int mgpu_piso_run(MgpuCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier) {
  if (!c || !ier) return MGPU_E_ARG;
  *ier = 0;
  if (nrec) *nrec = 0;
  if (!c->ctrl.transient) {
    *ier = 30;
    return 0;
  }
  if (c->ctrl.dt <= 0.0) {
    *ier = 31;
    return 0;
  }
  int n_steps = std::max(1, c->ctrl.n_time_max);
  if (nsteps > 0) n_steps = std::min(n_steps, nsteps);
  TRY(ensure_recs(c, n_steps + 1));
  TRY(begin_run(c));
  TRY(reset_status(c, 1, n_steps + 1));
  TRY(launch_fill(c->d.apc, c->d.N, 1.0, c->stream));
  TRY(launch_gradients(c->d, c->P, c->stream));
  TRY(launch_rhiechow(c->d, c->P, c->stream));
  c->launches += 3;
  for (int it = 0; it < n_steps; ++it) {
    TRY(outer_iteration(c, true));
    if ((it + 1) % 64 == 0 && it + 1 < n_steps) {
      int ab = 0;
      MGPU_CUDA(cudaMemcpyAsync(&ab, &c->d.st->abort, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
      MGPU_CUDA(cudaStreamSynchronize(c->stream));
      if (ab) break;
    }
  }
  return end_run(c, n_steps, log, logcap, nrec, ier);
}

int mgpu_pimple_run(MgpuCase* c, int nsteps, MgpuIterRec* log, int logcap, int* nrec, int* ier) {
  if (!c || !ier) return MGPU_E_ARG;
  *ier = 0;
  if (nrec) *nrec = 0;
  if (!c->ctrl.transient) {
    *ier = 50;
    return 0;
  }
  if (c->ctrl.dt <= 0.0) {
    *ier = 51;
    return 0;
  }
  int n_steps = std::max(1, c->ctrl.n_time_max);
  if (nsteps > 0) n_steps = std::min(n_steps, nsteps);
  TRY(ensure_recs(c, n_steps + 1));
  TRY(begin_run(c));
  c->P.pimple = 1;
  TRY(reset_status(c, 1, n_steps + 1));
  TRY(launch_fill(c->d.apc, c->d.N, 1.0, c->stream));
  TRY(launch_gradients(c->d, c->P, c->stream));
  TRY(launch_rhiechow(c->d, c->P, c->stream));
  c->launches += 3;
  int e = 0;
  for (int it = 0; it < n_steps && !e; ++it) {
    e = pimple_step(c);
    if (!e && (it + 1) % 64 == 0 && it + 1 < n_steps) {
      int ab = 0;
      if (cudaMemcpyAsync(&ab, &c->d.st->abort, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
          cudaStreamSynchronize(c->stream) != cudaSuccess) {
        e = cuda_fail(cudaGetLastError(), "status read", __FILE__, __LINE__);
        break;
      }
      if (ab) break;
    }
  }
  c->P.pimple = 0;
  if (e) return e;
  return end_run(c, n_steps, log, logcap, nrec, ier);
}

int mgpu_nan_scan(MgpuCase* c, int* ifin, int* field, int* cell, double* val, int* kind) {
  if (!c || !ifin || !field || !cell || !val || !kind) return MGPU_E_ARG;
  TRY(reset_status(c, 0, 1));
  TRY(launch_diag(c->d, c->P, 0, c->stream));
  DevStatus h{};
  MGPU_CUDA(cudaMemcpyAsync(&h, c->d.st, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  MGPU_CUDA(cudaStreamSynchronize(c->stream));
  *ifin = h.ier == 60 ? 1 : 0;
  *field = h.nan_field;
  *cell = h.nan_cell;
  *val = h.nan_val;
  *kind = h.nan_kind;
  return 0;
}

int mgpu_case_stage(MgpuCase* c, int what, int ts_order, const double* apc, double* aval, double* rhs, double* ap,
                    const double* pp) {
  if (!c || what < 0 || what > 7 || (what == 7 && !c->d.energy)) return MGPU_E_ARG;
  DeviceCase& d = c->d;
  cudaStream_t s = c->stream;
  const long N = d.N;
  TRY(reset_status(c, ts_order, 1));
  if (apc) MGPU_CUDA(cudaMemcpyAsync(d.apc, apc, sizeof(double) * N, cudaMemcpyHostToDevice, s));
  if (what == 0) {
    TRY(launch_gradients(d, c->P, s));
  } else if (what <= 3) {
    if (c->P.conv_blend > 0.0) {
      TRY(launch_limiter(d, c->P, what - 1, s));
      TRY(launch_momentum(d, c->P, what - 1, s));
    } else {  // the path a run takes
      TRY(launch_mom_interior(d, c->P, s));
      TRY(launch_mom_finish(d, c->P, what - 1, s));
    }
  } else if (what == 4) {
    TRY(launch_rhiechow(d, c->P, s));
  } else if (what == 5) {
    TRY(launch_ppe(d, c->P, s));
  } else if (what == 7) {
    TRY(launch_temperature(d, c->P, s));
  } else {
    if (!pp) return MGPU_E_ARG;
    MGPU_CUDA(cudaMemcpyAsync(d.pp, pp, sizeof(double) * N, cudaMemcpyHostToDevice, s));
    // af of the last PPE assembly is reused by the flux correction
    TRY(launch_correct(d, c->P, s));
  }
  MGPU_CUDA(cudaStreamSynchronize(s));
  const double* A = (what == 5) ? d.pval : d.aval;
  const bool rows = (what >= 1 && what <= 5) || what == 7;
  if (aval && rows) TRY(copy_sync(aval, A, sizeof(double) * d.nnz, cudaMemcpyDeviceToHost, c->stream));
  if (rhs && rows) TRY(copy_sync(rhs, d.rhs, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
  if (ap && ((what >= 1 && what <= 3) || what == 7))
    TRY(copy_sync(ap, d.ap, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
  return 0;
}

int mgpu_temperature_upload(MgpuCase* c, const double* T, const double* T_old, const double* T_old_old) {
  if (!c || !T) return MGPU_E_ARG;
  DeviceCase& d = c->d;
  const size_t bytes = sizeof(double) * (size_t)d.N;
  MGPU_CUDA(cudaMemcpyAsync(d.T, T, bytes, cudaMemcpyHostToDevice, c->stream));
  if (d.energy) {
    if (T_old)
      MGPU_CUDA(cudaMemcpyAsync(d.T_old, T_old, bytes, cudaMemcpyHostToDevice, c->stream));
    else
      MGPU_CUDA(cudaMemcpyAsync(d.T_old, d.T, bytes, cudaMemcpyDeviceToDevice, c->stream));
    if (T_old_old)
      MGPU_CUDA(cudaMemcpyAsync(d.T_old_old, T_old_old, bytes, cudaMemcpyHostToDevice, c->stream));
    else
      MGPU_CUDA(cudaMemcpyAsync(d.T_old_old, d.T, bytes, cudaMemcpyDeviceToDevice, c->stream));
  }
  MGPU_CUDA(cudaStreamSynchronize(c->stream));
  return 0;
}

int mgpu_temperature_download(MgpuCase* c, double* T, double* gt) {
  if (!c) return MGPU_E_ARG;
  DeviceCase& d = c->d;
  const long N = d.N;
  if (T) TRY(copy_sync(T, d.T, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
  if (gt) {
    if (!d.energy) {
      std::memset(gt, 0, sizeof(double) * 3 * N);
    } else {
      std::vector<double> planes(3 * N);
      TRY(copy_sync(planes.data(), d.gt, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, c->stream));
      for (long i = 0; i < N; ++i)
        for (int k = 0; k < 3; ++k) gt[3 * i + k] = planes[k * N + i];
    }
  }
  return 0;
}

int mgpu_interface_set(MgpuCase* c, int n, const int32_t* faces, const double* u, const double* p) {
  if (!c || n < 0 || (n > 0 && !faces)) return MGPU_E_ARG;
  if (c->d.n_iface == 0) {
    set_error("mgpu_interface_set: the case has no interface zone");
    return MGPU_E_ARG;
  }
  if (n == 0 || (!u && !p)) return 0;
  std::vector<int> f0(n);
  for (int k = 0; k < n; ++k) {
    if (faces[k] < 1 || faces[k] > c->d.F) {
      set_error("mgpu_interface_set: face index out of range");
      return MGPU_E_ARG;
    }
    f0[k] = faces[k] - 1;
  }
  cudaStream_t s = c->stream;
  int* df = nullptr;
  double *du = nullptr, *dp = nullptr;
  MGPU_CUDA(cudaMallocAsync((void**)&df, sizeof(int) * n, s));
  if (u) MGPU_CUDA(cudaMallocAsync((void**)&du, sizeof(double) * 3 * n, s));
  if (p) MGPU_CUDA(cudaMallocAsync((void**)&dp, sizeof(double) * n, s));
  MGPU_CUDA(cudaMemcpyAsync(df, f0.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
  if (u) MGPU_CUDA(cudaMemcpyAsync(du, u, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
  if (p) MGPU_CUDA(cudaMemcpyAsync(dp, p, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  k_iface_scatter<<<ceil_div(n, 256), 256, 0, s>>>(n, df, du, dp, c->d.F, c->d.iface_vel, c->d.iface_p);
  MGPU_LAUNCH_CHECK("k_iface_scatter");
  cudaFreeAsync(df, s);
  if (du) cudaFreeAsync(du, s);
  if (dp) cudaFreeAsync(dp, s);
  MGPU_CUDA(cudaStreamSynchronize(s));
  return 0;
}

int mgpu_interface_set_T(MgpuCase* c, int n, const int32_t* faces, const double* T, const double* q,
                         const int32_t* mode) {
  if (!c || n < 0 || (n > 0 && !faces)) return MGPU_E_ARG;
  if (c->d.n_iface == 0 || !c->d.energy) {
    set_error("mgpu_interface_set_T: the case has no interface zone or no energy equation");
    return MGPU_E_ARG;
  }
  if (n == 0 || (!T && !q && !mode)) return 0;
  std::vector<int> f0(n);
  for (int k = 0; k < n; ++k) {
    if (faces[k] < 1 || faces[k] > c->d.F || (mode && mode[k] != 0 && mode[k] != 1)) {
      set_error("mgpu_interface_set_T: face index or mode out of range");
      return MGPU_E_ARG;
    }
    f0[k] = faces[k] - 1;
  }
  cudaStream_t s = c->stream;
  int *df = nullptr, *dm = nullptr;
  double *dT = nullptr, *dq = nullptr;
  MGPU_CUDA(cudaMallocAsync((void**)&df, sizeof(int) * n, s));
  if (T) MGPU_CUDA(cudaMallocAsync((void**)&dT, sizeof(double) * n, s));
  if (q) MGPU_CUDA(cudaMallocAsync((void**)&dq, sizeof(double) * n, s));
  if (mode) MGPU_CUDA(cudaMallocAsync((void**)&dm, sizeof(int) * n, s));
  MGPU_CUDA(cudaMemcpyAsync(df, f0.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
  if (T) MGPU_CUDA(cudaMemcpyAsync(dT, T, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  if (q) MGPU_CUDA(cudaMemcpyAsync(dq, q, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  if (mode) MGPU_CUDA(cudaMemcpyAsync(dm, mode, sizeof(int) * n, cudaMemcpyHostToDevice, s));
  k_iface_scatter_T<<<ceil_div(n, 256), 256, 0, s>>>(n, df, dT, dq, dm, c->d.iface_T, c->d.iface_q,
                                                     c->d.iface_tmode);
  MGPU_LAUNCH_CHECK("k_iface_scatter_T");
  cudaFreeAsync(df, s);
  if (dT) cudaFreeAsync(dT, s);
  if (dq) cudaFreeAsync(dq, s);
  if (dm) cudaFreeAsync(dm, s);
  MGPU_CUDA(cudaStreamSynchronize(s));
  return 0;
}

int mgpu_interface_mode(MgpuCase* c, int p_dirichlet) {
  if (!c) return MGPU_E_ARG;
  c->d.iface_pdir = p_dirichlet ? 1 : 0;
  return 0;
}

int mgpu_interface_extract(MgpuCase* c, int cap, int32_t* faces, double* u, double* p, double* T, int* n) {
  if (!c || !n) return MGPU_E_ARG;
  const int m = (int)c->iface_faces.size();
  *n = m;
  if (m == 0 || cap <= 0) return 0;
  const int k = std::min(m, cap);
  cudaStream_t s = c->stream;
  double* out = nullptr;
  MGPU_CUDA(cudaMallocAsync((void**)&out, sizeof(double) * 5 * k, s));
  k_iface_gather<<<ceil_div(k, 256), 256, 0, s>>>(k, c->d_iface_faces, c->d.c0, c->d.u, c->d.p, c->d.T, c->d.N,
                                                  out);
  MGPU_LAUNCH_CHECK("k_iface_gather");
  std::vector<double> h(5 * (size_t)k);
  MGPU_CUDA(cudaMemcpyAsync(h.data(), out, sizeof(double) * 5 * k, cudaMemcpyDeviceToHost, s));
  cudaFreeAsync(out, s);
  MGPU_CUDA(cudaStreamSynchronize(s));
  for (int j = 0; j < k; ++j) {
    if (faces) faces[j] = c->iface_faces[j] + 1;
    if (u)
      for (int q = 0; q < 3; ++q) u[3 * j + q] = h[5 * j + q];
    if (p) p[j] = h[5 * j + 3];
    if (T) T[j] = h[5 * j + 4];
  }
  return 0;
}

int mgpu_case_timing(const MgpuCase* c, MgpuTiming* t) {
  if (!c || !t) return MGPU_E_ARG;
  *t = c->timing;
  return 0;
}

int mgpu_case_solve_times(const MgpuCase* c, double* ms, int cap, int* n) {
  if (!c || !n) return MGPU_E_ARG;
  const int m = (int)(c->ev_used / 2);
  *n = m;
  for (int i = 0; i < m && i < cap && ms; ++i) {
    float t = 0.f;
    cudaEventElapsedTime(&t, c->ev_pool[2 * i], c->ev_pool[2 * i + 1]);
    ms[i] = t;
  }
  return 0;
}

int mgpu_case_set_profiling(MgpuCase* c, int on) {
  if (!c) return MGPU_E_ARG;
  c->profiling = on ? 1 : 0;
  return 0;
}

}  // extern "C"
