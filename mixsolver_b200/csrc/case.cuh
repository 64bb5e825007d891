// case.cuh -- device-resident state of one SIMPLE/PISO case.
#pragma once

#include <vector>

#include "common.cuh"

namespace mgpu {

// Run status shared by every kernel of a run. A kernel returns at once when
// `abort` is set, which gives the reference's early returns (ier /= 0,
// convergence) without a host round trip per outer iteration.
struct DevStatus {
  int abort;      // set on ier /= 0 or convergence
  int ier;        // reference driver code (20, 21, 33, 34, 60, ...)
  int cur_it;     // 0-based index of the outer iteration / step in progress
  int converged;
  int timeout;    // a bounded grid barrier ran out
  int ts_order;   // 0 steady, 1 Euler, 2 BDF2 (fields_t%ts_order)
  int nan_field, nan_cell;
  int nan_kind;
  int it_limit;  // > 0: the run ends (abort, no ier) once cur_it reaches it
  double nan_val;
  double t_now;
  unsigned long long imbal_bits, du_bits, umax_bits;  // max-reductions (bit patterns of x >= 0)
  unsigned long long dT_bits;                          // max |T - T before its solve|
  unsigned long long nan_key;                          // min (cell*5+field), fields u, v, w, p, T
  // solves of the earlier outer iterations of a PIMPLE step: largest
  // iteration count, sum of the momentum residuals (in solve order)
  int acc_itl;
  double acc_res;
  unsigned spin_limit;  // polls before a bounded barrier wait gives up (0: the default, ~2 s)
  unsigned poll_ns;     // sleep between a barrier wait's polls (0: poll back to back)
};

// Krylov solve arguments (matrix, preconditioner data, work, result slot).
struct KrylovArgs {
  int n;
  const int* row_ptr;
  const int* col;
  const int* diag;
  const double* aval;
  double* fval;  // ILU(0)/IC(0) factor values (same pattern)
  const double* b;
  double* x;
  double *r, *r0, *p, *v, *s, *t, *ph, *sh, *z, *w;
  int nlev_lo;
  const int* lo_ptr;
  const int* lo_rows;
  int nlev_up;
  const int* up_ptr;
  const int* up_rows;
  const int* lt_ptr;  // transposed strictly-lower part, per column k: rows i > k (descending)
  const int* lt_pos;  // position of L(i,k) in row i
  double tol;
  int maxit;
  int precond;  // 0 ILU0, 1 Jacobi, 2 IC0
  int zero_x;   // x := 0 before the solve (pressure correction)
  int mpi_mode; // 1: the one-rank distributed solver variants (mod_uns_linsolver_mpi.f90)
  double* partials;  // 4 * gridDim doubles
  unsigned long long* bar;  // grid-barrier arrival counter (zeroed before each launch)
  DevStatus* st;
  MgpuIterRec* recs;
  int slot;            // record slot of this solve
  int ier_breakdown;   // driver code when ierr == 2 (0: none)
  int* ferr;           // factorisation status written by the factor kernel
  int sweep_threads;   // threads of a sync-free triangular sweep (set at launch)
  int sweep_sleep;     // nanosleep of a long wait in that sweep (0: spin)
};

// Data of a polynomial-preconditioned solve in working precision V: the
// matrix copy and inverse diagonal in V, work vectors in V (10 N), inner
// relative tolerance. V = float is the mixed-precision form (FP32 inner
// Krylov inside FP64 refinement); V = double the same algorithms in FP64.
template <typename V>
struct MixedArgsT {
  V* a32;
  V* dinv;
  V* w32;
  double tau;
  int cheb_k;        // Chebyshev-Jacobi degree of the pressure preconditioner (<= 1: Jacobi)
  double cheb_ratio; // lambda_max / lambda_min of the Chebyshev interval
  int ell_w;         // ELL width (max entries per row) when ell_col is set
  const int* ell_col;  // column-major ELL columns, W*ell_ld (padding: the row itself)
  V* ell_val;          // values in the same layout (padding: 0)
  double* red;         // chunk reduction partials: mixed_red_words(N) doubles
  int pf;              // 1: each SpMV tile prefetches the next tile's ELL entries into L2
  double rel_delta;    // FP64 polynomial PCG: replace the recursive residual once its norm fell by this factor (0: only to confirm convergence)
  int ell_ld;    // leading dimension of the ELL arrays: N rounded up to a multiple of 4
  // single-system grid launches: chunk-sum slots per sum a block keeps in its
  // dynamic shared memory (set at launch; 0 elsewhere)
  int cp_slots;
  // the mixed form's PCG (V = float): the FP64 values in the ELL layout, for
  // the FP64 conjugate-gradient product q = A p (null: the CSR values)
  double* ell64;
};
using MixedArgs = MixedArgsT<float>;

// Device bytes a mixed solve keeps live per row: ELL columns, FP32 and FP64
// values, the FP32 work vectors and inverse diagonal, and the FP64 vectors
// (x, b, the residual, two search directions, q).
inline double mixed_row_bytes(int ell_w) { return 16.0 * ell_w + 4.0 * 5 + 8.0 * 6; }

// The mixed-precision solves reduce over fixed row chunks (32 rows) and
// super-chunks (256 rows), so their results do not depend on how rows are
// spread over blocks. Work words of those partials for n rows: two halves of
// two sums each.
#ifndef MGPU_MIXED_MAX_ROWS_LOG2
#define MGPU_MIXED_MAX_ROWS_LOG2 23
#endif
#ifndef MGPU_BLOCK_MAX_ROWS
#define MGPU_BLOCK_MAX_ROWS 32768
#endif
constexpr int kMixedMaxRows = 1 << MGPU_MIXED_MAX_ROWS_LOG2;
constexpr int kSuperRows = 256;
constexpr int kBlockMaxRows = MGPU_BLOCK_MAX_ROWS;  // rows one block of a mixed solve may hold
inline long mixed_red_words(long n) { return 4l * ((n + kSuperRows - 1) / kSuperRows); }

// One system of a batched solve.
struct alignas(16) BatchSys {
  KrylovArgs a;
  MixedArgs m;
};

// A lane of a batched launch: nblocks co-resident blocks that solve systems
// one after the other, taken from the queue of its width class (cls) and,
// once that is empty, from the queues of narrower classes.
struct BatchLane {
  int first_block, nblocks, cls, pad;
};

// Device tables of one batched Krylov launch.
struct LanePlan {
  const BatchSys* sys;
  const BatchLane* lanes;
  const int* block_lane;
  const int* q_items;         // systems of every class queue, longest first
  const int* q_start;         // class c's queue: q_items[q_start[c] .. q_start[c + 1])
  int* q_head;                // next position of each class queue (zeroed per launch)
  int* lane_slot;             // two slots per lane: the system its blocks run next
  unsigned long long* bars;   // one barrier counter per lane
  double* partials;           // 8 doubles per block
  unsigned long long* lane_t; // optional: start and end time (ns) of each lane
  int ncls, nlanes, nblocks;
};

struct DeviceCase {
  int N = 0, F = 0, nnz = 0;
  // faces
  int *c0 = nullptr, *c1 = nullptr, *fgrp = nullptr;
  double *xf = nullptr, *sf = nullptr, *area = nullptr, *lf = nullptr;  // xf,sf: 3 SoA planes
  // cells
  double *vol = nullptr, *xc = nullptr;  // xc: 3 SoA planes
  int *cf_ptr = nullptr, *cf = nullptr, *cf_slot = nullptr;
  // per cell-face entry: 1 when no earlier entry of the cell has the same CSR
  // slot (two faces between the same two cells share one), so the assembly
  // writes the slot instead of adding to it
  unsigned char* cf_first = nullptr;
  // energy equation: T (N), its history, gradient (3 planes of N), T before
  // the solve, limiter (conv_blend > 0); energy: the equation is solved
  double *T = nullptr, *T_old = nullptr, *T_old_old = nullptr, *gt = nullptr, *Tprev = nullptr,
         *psiT = nullptr;
  int energy = 0;
  // per-face constants (bit-identical to recomputing them in the face loops)
  double *dn = nullptr;   // interior |xc1-xc0|, boundary |xf-xc0|
  double *dsf = nullptr;  // interior (xc1-xc0).sf
  double *Dm = nullptr;   // momentum diffusion coefficient
  double *tv = nullptr;   // 3 planes: sf - dvec*(area^2/sd)
  double *mnc = nullptr;  // nonorth_corr*mu_f
  // CSR pattern and level sets
  int *row_ptr = nullptr, *col = nullptr, *diag = nullptr;
  int nlev_lo = 0, nlev_up = 0;
  int *lo_ptr = nullptr, *lo_rows = nullptr, *up_ptr = nullptr, *up_rows = nullptr;
  int *lt_ptr = nullptr, *lt_pos = nullptr;
  DevGroup* groups = nullptr;
  int ngroups = 0;
  // outflow rescale (cases with an outflow zone): fixed-flux boundary faces and
  // outflow faces, each list in face order
  int *of_req = nullptr, *of_out = nullptr;
  int n_of_req = 0, n_of_out = 0;
  // momentum: each cell's boundary faces with a group (face order) and the
  // interior sums of the three components (ap, rhs per component)
  int *bf_ptr = nullptr, *bf = nullptr;
  double *mom_ap = nullptr, *mom_rhs = nullptr;
  // fields (SoA)
  double *u = nullptr, *p = nullptr, *gp = nullptr, *gu = nullptr, *flux = nullptr, *apc = nullptr;
  double *ap = nullptr, *rhs = nullptr, *pp = nullptr, *uo = nullptr, *u_old = nullptr, *u_old_old = nullptr;
  double *psi = nullptr, *af = nullptr;
  double *aval = nullptr, *pval = nullptr, *fval = nullptr;
  float *a32 = nullptr, *dinv32 = nullptr, *w32 = nullptr;  // mixed-precision form
  int* ell_col = nullptr;  // column-major ELL pattern of the FP32 copy (W*N)
  float* ell_val = nullptr;
  double *a64 = nullptr, *dinv64 = nullptr, *w64 = nullptr, *ell_val64 = nullptr;  // FP64 polynomial form
  int ell_w = 0;
  int ell_ld = 0;  // ELL leading dimension: N rounded up to a multiple of 4
  double* red32 = nullptr;  // chunk reduction partials of the mixed-precision solves
  // Krylov work
  double *kw = nullptr;  // 10*N
  double* partials = nullptr;
  unsigned long long* bar = nullptr;
  int* ferr = nullptr;
  DevStatus* st = nullptr;
  MgpuIterRec* recs = nullptr;
  int rec_cap = 0;
  double* ramp = nullptr;  // inlet-speed and pressure-value ramp factors in effect (2)
  // coupling interface (cases with interface zones): the peer's face velocity
  // (3 planes of F) and face pressure (F), and the interface mode
  double *iface_vel = nullptr, *iface_p = nullptr;
  int n_iface = 0;     // interface faces
  int iface_pdir = 0;  // 1: pressure is the interface constraint (g_iface_p_dir)
  // the peer's face temperature and heat flux (F each) and the per-face mode
  // (0 Dirichlet, 1 Neumann), interface cases only
  double *iface_T = nullptr, *iface_q = nullptr;
  int* iface_tmode = nullptr;
};

// Launch helpers implemented in the .cu files.
int launch_krylov_bicgstab(const KrylovArgs& a, cudaStream_t s);
int launch_krylov_pcg(const KrylovArgs& a, cudaStream_t s);
int launch_factor(const KrylovArgs& a, int kind, cudaStream_t s);
int krylov_grid(int n, int& block, int which);
int launch_pcg_mixed(const KrylovArgs& a, const MixedArgs& m, cudaStream_t s);
int launch_bicgstab_mixed(const KrylovArgs& a, const MixedArgs& m, cudaStream_t s);
int launch_pcg_poly64(const KrylovArgs& a, const MixedArgsT<double>& m, cudaStream_t s);
int launch_bicgstab_poly64(const KrylovArgs& a, const MixedArgsT<double>& m, cudaStream_t s);
int batch_capacity(bool pcg, int ell);  // ell: 0 CSR, 1 ELL, 2 ELL + L2 prefetch
int launch_mixed_batch(const LanePlan& p, bool pcg, int ell, cudaStream_t s);
int launch_spmv(int n, const int* rp, const int* col, const double* val, const double* x, double* y,
                cudaStream_t s);

}  // namespace mgpu
