// krylov_poly.cuh -- the Krylov bodies of the mixed-precision form, templated
// on the working precision V of the inner Krylov vectors and matrix copy.
// V = float is the mixed-precision form (krylov_mixed.cu); V = double runs
// the same algorithms in FP64 throughout (krylov_poly64.cu), which isolates
// what the FP32 arithmetic buys.
//
// FP64 iterative refinement around an FP32 inner Krylov method:
//   r = b - A x                      (FP64 SpMV, FP64 accumulation)
//   solve A d = r / |r| to tau        (FP32 matrix and vectors, FP32 SpMV
//                                      accumulation, Jacobi or Chebyshev-Jacobi
//                                      preconditioner in FP32; every dot
//                                      product and norm in FP64)
//   x += |r| d                        (FP64)
// until |b - A x| / |b| <= tol (the true residual, recomputed in FP64). The
// matrix is rounded to FP32 inside the same launch; `it` counts inner
// iterations. The pressure PCG runs by default with reliable updates instead
// (MixedArgs::reliable): one FP32 CG stream whose steps go straight into the
// FP64 x, with the FP32 residual replaced by the FP64 b - A x every time it
// has fallen by a fixed factor, so no refinement step restarts the Krylov
// space (pcg_reliable).
//
// Layout independence. A solve runs on a group of co-resident blocks (the
// whole grid of a single-system launch, or one lane of a batched launch).
// Every row's arithmetic is its own (FP32 SpMV in CSR order, element-wise
// updates), and every sum is taken over fixed row chunks: the 32 values of a
// 32-row chunk in a fixed butterfly, the 8 chunk sums of a 256-row
// super-chunk in index order, super-chunks l, l + 32, ..., l + 224 of a group
// of 256 in order, the 32 lane sums in a butterfly, the group sums in order. Rows go to blocks in grid-stride tiles of whole
// super-chunks. So a system's result is the same bit for bit whatever the
// number of blocks, the block size, or the other systems in the launch.
//
// This form does not reproduce the reference's iteration counts (different
// preconditioner, different precision); it converges the same systems to the
// same tolerance on the true residual.
#pragma once

#include <algorithm>
#include <type_traits>

#include "persist.cuh"

namespace mgpu {
namespace {

__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double vfma(double a, double b, double c) { return fma(a, b, c); }

// ---------------------------------------------------------------------------
// rows and layout-independent sums
// ---------------------------------------------------------------------------

// The rows of one block, in tiles of blockDim.x rows: tile t of the group at
// rows [t * blockDim.x, (t + 1) * blockDim.x) for t = rank, rank + nb, ...,
// so all blocks stream the same narrow window of every array at a time.
// Tiles are whole super-chunks (blockDim.x is a multiple of kSuperRows), so
// the layout-independent sums see the same super-chunks on any grid.
struct Rows {
  int start;   // first row of this block's first tile
  int stride;  // rows between its consecutive tiles
  int n;       // end of the rows (exclusive)
};

// A block holds at most kBlockMaxRows rows (the chunk sums of its tiles live
// in shared memory); launches and lane plans size their groups accordingly,
// and a group too small for its system refuses it (fits_group).
__device__ __forceinline__ bool fits_group(int n, const VGrid& g) {
  const long stride = (long)g.nb * blockDim.x;
  return ((n + stride - 1) / stride) * (long)blockDim.x <= kBlockMaxRows;
}

// The chunk-sum slots the launch gave a block (DYN kernels) hold its tiles.
__device__ __forceinline__ bool fits_slots(int n, const VGrid& g, int cp_slots) {
  const long bd = blockDim.x;
  const long tiles = ((long)n + g.nb * bd - 1) / (g.nb * bd);
  return tiles * (bd / 32) <= cp_slots;
}

__device__ __forceinline__ Rows block_rows(int n, const VGrid& g) {
  return Rows{g.rank * (int)blockDim.x, g.nb * (int)blockDim.x, n};
}

// Reduction state of one system. Chunk sums (a fixed butterfly over the 32
// rows of a warp) stay in the block's shared memory (only the owning block
// reads them); super-chunk sums (the 8 chunk sums in order) go to global memory in
// two halves that consecutive reductions alternate, so a block running ahead
// into the next reduction cannot overwrite values a slower block still reads.
struct Red {
  double* base;  // 2 halves x 2 sums x nsc super-chunk sums
  int nsc, half;
  double* cp;    // the block's chunk sums in shared memory: sum q of chunk j at cp[q * cps + j]
  int cps;
  __device__ double* sp() const { return base + (half ? 2l * nsc : 0); }
};

// per block: chunk sums (rows of a block <= kBlockMaxRows) and level sums
constexpr int kBlockMaxChunks = kBlockMaxRows / 32;
constexpr int kMaxGroups = (kMixedMaxRows / kSuperRows + 255) / 256;  // groups of 256 super-chunks
__shared__ double s_cp[2][kBlockMaxChunks];
__shared__ double lvg[2][kMaxGroups];

// The dynamic shared memory of a single-system grid launch: the block's chunk
// sums, 2 x MixedArgsT::cp_slots doubles, sized at launch for the rows the
// block owns.
extern __shared__ __align__(16) unsigned char mixed_dyn[];

// DYN: the chunk sums live in the launch's dynamic shared memory (single-system
// grid kernels); otherwise in the static array sized for kBlockMaxRows rows
// (single-block kernels, batched lanes).
template <typename V, bool DYN>
__device__ __forceinline__ Red make_red(const MixedArgsT<V>& m, int n) {
  if constexpr (DYN)
    return Red{m.red, (n + kSuperRows - 1) / kSuperRows, 0, reinterpret_cast<double*>(mixed_dyn), m.cp_slots};
  else
    return Red{m.red, (n + kSuperRows - 1) / kSuperRows, 0, &s_cp[0][0], kBlockMaxChunks};
}

// Sum this thread's row values c[q] (zero for rows past n) over the warp's
// 32 rows of the tile starting at base into the tile's chunk slot. Every lane
// of the warp calls it.
template <int NQ>
__device__ __forceinline__ void red_put(const Red& R, const Rows& rows, int base, const double (&c)[NQ]) {
  double s[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) s[q] = warp_sum(c[q]);
  if ((threadIdx.x & 31) == 0 && base < rows.n) {
    const int slot = ((base - rows.start) / rows.stride) * (blockDim.x >> 5) + (threadIdx.x >> 5);
#pragma unroll
    for (int q = 0; q < NQ; ++q) R.cp[q * R.cps + slot] = s[q];
  }
}

// Finish a reduction: super-chunk sums of this block's rows, group barrier,
// then every block forms the total from the super-chunk sums in the same fixed
// tree. Returns false when the barrier wait ran out.
// Finish a reduction: super-chunk sums of this block's tiles, group barrier,
// then every block forms the total from the super-chunk sums in the same fixed
// tree: in a group of 256 super-chunks lane l adds super-chunks l, l + 32, ...,
// l + 224 in that order, the 32 lanes meet in a butterfly, and the group sums
// are added in order. Returns false when the barrier wait ran out.
template <int NQ, bool L1>
__device__ __forceinline__ bool red_total(Red& R, const Rows& rows, VGrid& g, DevStatus* st, double (&out)[NQ]) {
  static_assert(NQ <= 2, "at most two sums per reduction");
  constexpr int kChunks = kSuperRows / 32;  // chunks per super-chunk
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double* sp = R.sp();
  const int nsc = R.nsc;
  __syncthreads();  // this block's chunk sums are in R.cp
  const int ntb = rows.start < rows.n ? (rows.n - rows.start + rows.stride - 1) / rows.stride : 0;
  const int per_tile = blockDim.x / kSuperRows;
  for (int pr = threadIdx.x; pr < ntb * per_tile; pr += blockDim.x) {
    const int sc = (rows.start + (pr / per_tile) * rows.stride) / kSuperRows + pr % per_tile;
    if (sc >= nsc) continue;  // a super-chunk past the last row
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const double* cq = R.cp + q * R.cps + pr * kChunks;
      double acc = cq[0];
#pragma unroll
      for (int j = 1; j < kChunks; ++j) acc = acc + cq[j];
      sp[(long)q * nsc + sc] = acc;
    }
  }
  if (g.nb > 1) {
    if (!vg_sync(g, st)) return false;
  } else {
    __syncthreads();
  }
  const int ng = (nsc + 255) >> 8;  // groups of 256 super-chunks
  for (int k = warp; k < ng; k += nw) {
    const int s0 = k * 256 + lane;
    double v[NQ][8];
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
      for (int r = 0; r < 8; ++r) v[q][r] = s0 + 32 * r < nsc ? ldv(&sp[(long)q * nsc + s0 + 32 * r]) : 0.0;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double acc = v[q][0];
#pragma unroll
      for (int r = 1; r < 8; ++r) acc = acc + v[q][r];
      acc = warp_sum(acc);
      if (lane == 0) lvg[q][k] = acc;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double acc = lvg[q][0];
    for (int k = 1; k < ng; ++k) acc = acc + lvg[q][k];
    out[q] = acc;
  }
  __syncthreads();  // the chunk sums and lvg are reused by the next reduction
  R.half ^= 1;
  return true;
}

// ---------------------------------------------------------------------------
// FP32 SpMV rows
// ---------------------------------------------------------------------------

// y = (A32 x)_i, FP32 accumulation in CSR order; the row's loads are issued
// before any accumulation.
template <typename V, bool L1, int MAXNZ>
__device__ __forceinline__ V spmv32_csr(const int* __restrict__ rp, const int* __restrict__ col,
                                            const V* __restrict__ val, const V* x, int i) {
  const int b = rp[i], e = rp[i + 1];
  V v[MAXNZ], xv[MAXNZ];
  int c[MAXNZ];
#pragma unroll
  for (int t = 0; t < MAXNZ; ++t)
    if (b + t < e) {
      c[t] = col[b + t];
      v[t] = val[b + t];
    }
#pragma unroll
  for (int t = 0; t < MAXNZ; ++t)
    if (b + t < e) xv[t] = ldv(&x[c[t]]);
  V acc = V(0);
#pragma unroll
  for (int t = 0; t < MAXNZ; ++t)
    if (b + t < e) acc = vfma(v[t], xv[t], acc);
  for (int k = b + MAXNZ; k < e; ++k) acc = vfma(val[k], ldv(&x[col[k]]), acc);
  return acc;
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Runs body(std::integral_constant<int, WC>{}) with WC the ELL width when it
// is one the passes are compiled for (5: tetrahedra and 2-D quadrilaterals,
// 7: hexahedra), else WC = 0 (the width read at run time); a compile-time
// width drops the per-entry width checks from every row of the pass.
template <int ELL, typename F>
__device__ __forceinline__ void with_width(int w, F&& body) {
  if constexpr (ELL == 0) {
    body(std::integral_constant<int, 0>{});
  } else {
    switch (w) {
      case 5:
        body(std::integral_constant<int, 5>{});
        break;
      case 7:
        body(std::integral_constant<int, 7>{});
        break;
      default:
        body(std::integral_constant<int, 0>{});
    }
  }
}

// kRows rows per thread in the SpMV passes: every row's loads are issued
// before any product, so a warp keeps kRows rows of gathers in flight.
#ifndef MGPU_KROWS
#define MGPU_KROWS 1
#endif
constexpr int kRows = MGPU_KROWS;

// The SpMV passes read the argument structs through references, which stay
// in kernel-parameter space (single-system kernels) or shared memory (the
// batched kernel): no register holds a field between uses.
// FULL: every row of the step is below n (no per-entry row check).
// What an FP32 SpMV pass reads, copied once per pass into registers from
// wherever the solve's arguments live (kernel parameters, or a batch's
// descriptor table in global memory); the restrict qualifiers tell the
// compiler that the pass's stores do not touch them, so no field is reloaded
// per row.
template <typename V>
struct Sp32 {
  int n, w;
  const int* __restrict__ ecol;
  const V* __restrict__ eval;
  const int* __restrict__ rp;
  const int* __restrict__ col;
  const V* __restrict__ a32;
  const V* __restrict__ dinv;
  int pf;  // rows from a tile to the tile whose ELL entries it prefetches into L2 (0: none)
  int ld;  // ELL leading dimension (entry t of row i at t * ld + i, below 2^31)
};

template <typename V>
__device__ __forceinline__ Sp32<V> sp32_of(const KrylovArgs& a, const MixedArgsT<V>& m, const Rows& rows) {
  return Sp32<V>{a.n,    m.ell_w, m.ell_col, m.ell_val, a.row_ptr, a.col, m.a32, m.dinv,
                 m.pf * kRows * rows.stride, m.ell_ld};
}

template <typename V, bool L1, int ELL, bool FULL, int WC = 0>
__device__ __forceinline__ void spmv32_rows(const Sp32<V>& S, const V* x, const int (&i)[kRows],
                                            const bool (&in0)[kRows], V (&y)[kRows]) {
  bool in[kRows];
#pragma unroll
  for (int r = 0; r < kRows; ++r) in[r] = FULL || in0[r];
  if constexpr (ELL) {
    constexpr int WMAX = WC ? WC : 8;  // WC: the ELL width known at compile time
    const int W = WC ? WC : S.w;
    V v[kRows][WMAX], xv[kRows][WMAX];
    int c[kRows][WMAX];
#pragma unroll
    for (int r = 0; r < kRows; ++r)
#pragma unroll
      for (int t = 0; t < WMAX; ++t)
        if (t < W && in[r]) {
          c[r][t] = S.ecol[t * S.ld + i[r]];
          v[r][t] = S.eval[t * S.ld + i[r]];
        }
    if constexpr (ELL == 2) {
      // the same rows of this block's next tile: DRAM -> L2 while this tile's
      // gathers wait (no registers held)
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int j = i[r] + S.pf;
        if (j < S.n) {
#pragma unroll
          for (int t = 0; t < WMAX; ++t)
            if (t < W) {
              prefetch_l2(S.ecol + t * S.ld + j);
              prefetch_l2(S.eval + t * S.ld + j);
            }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kRows; ++r)
#pragma unroll
      for (int t = 0; t < WMAX; ++t)
        if (t < W && in[r]) xv[r][t] = ldv(&x[c[r][t]]);
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      V acc = V(0);
#pragma unroll
      for (int t = 0; t < WMAX; ++t)
        if (t < W && in[r]) acc = vfma(v[r][t], xv[r][t], acc);
      y[r] = acc;
    }
  } else {
#pragma unroll
    for (int r = 0; r < kRows; ++r) y[r] = in[r] ? spmv32_csr<V, L1, 8>(S.rp, S.col, S.a32, x, i[r]) : V(0);
  }
}

// y = A (z + beta pold) with each gathered entry formed as the owner row forms
// its new search direction (first: y = A z): the product of the new direction
// computed directly, from vectors no block writes during the pass.
template <typename V, bool L1, int ELL, bool FULL, int WC = 0>
__device__ __forceinline__ void spmv32_rows_dir(const Sp32<V>& S, const V* z, const V* pold, V beta, bool first,
                                                const int (&i)[kRows], const bool (&in0)[kRows], V (&y)[kRows]) {
  bool in[kRows];
#pragma unroll
  for (int r = 0; r < kRows; ++r) in[r] = FULL || in0[r];
  if constexpr (ELL) {
    constexpr int WMAX = WC ? WC : 8;  // WC: the ELL width known at compile time
    const int W = WC ? WC : S.w;
    V v[kRows][WMAX], xv[kRows][WMAX];
    int c[kRows][WMAX];
#pragma unroll
    for (int r = 0; r < kRows; ++r)
#pragma unroll
      for (int t = 0; t < WMAX; ++t)
        if (t < W && in[r]) {
          c[r][t] = S.ecol[t * S.ld + i[r]];
          v[r][t] = S.eval[t * S.ld + i[r]];
        }
    if constexpr (ELL == 2) {
      // the same rows of this block's next tile: DRAM -> L2 while this tile's
      // gathers wait (no registers held)
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int j = i[r] + S.pf;
        if (j < S.n) {
#pragma unroll
          for (int t = 0; t < WMAX; ++t)
            if (t < W) {
              prefetch_l2(S.ecol + t * S.ld + j);
              prefetch_l2(S.eval + t * S.ld + j);
            }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kRows; ++r)
#pragma unroll
      for (int t = 0; t < WMAX; ++t)
        if (t < W && in[r]) xv[r][t] = first ? ldv(&z[c[r][t]]) : vfma(beta, ldv(&pold[c[r][t]]), ldv(&z[c[r][t]]));
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      V acc = V(0);
#pragma unroll
      for (int t = 0; t < WMAX; ++t)
        if (t < W && in[r]) acc = vfma(v[r][t], xv[r][t], acc);
      y[r] = acc;
    }
  } else {
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      V acc = V(0);
      if (in[r]) {
        const int e = S.rp[i[r] + 1];
        for (int k = S.rp[i[r]]; k < e; ++k) {
          const int cc = S.col[k];
          const V x = first ? ldv(&z[cc]) : vfma(beta, ldv(&pold[cc]), ldv(&z[cc]));
          acc = vfma(S.a32[k], x, acc);
        }
      }
      y[r] = acc;
    }
  }
}

template <bool L1>
__device__ __forceinline__ double row_spmv64(const KrylovArgs& a, const double* x, int i) {
  double y = 0.0;
  const int e = a.row_ptr[i + 1];
  for (int k = a.row_ptr[i]; k < e; ++k) y = fma(a.aval[k], ldv(&x[a.col[k]]), y);
  return y;
}

__device__ void write_result_m(const KrylovArgs& a, const VGrid& g, int it, double res, int ierr) {
  if (g.rank == 0 && threadIdx.x == 0) {
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

// Loop over this block's rows in tiles of blockDim.x: every thread runs the
// same number of tiles (rows past the range are masked), so warp-wide sums in
// the body are safe.
#define MGPU_TILES(rows, base) for (int base = (rows).start; base < (rows).n; base += (rows).stride)
// The same over kRows tiles per step: rows base + r * stride + threadIdx.x.
#define MGPU_STEPS(rows, base) for (int base = (rows).start; base < (rows).n; base += kRows * (rows).stride)
// A step body instantiated twice: FULL = true when all kRows tiles of the
// step lie below n (the uniform case), false for the last, partial step.
#define MGPU_SPLIT_FULL(rows, base, FULL, ...)                                            \
  if ((base) + (kRows - 1) * (rows).stride + (int)blockDim.x <= (rows).n) {              \
    constexpr bool FULL = true;                                                            \
    __VA_ARGS__                                                                            \
  } else {                                                                                 \
    constexpr bool FULL = false;                                                           \
    __VA_ARGS__                                                                            \
  }
#define MGPU_STEP_ROWS(rows, base, i, in)          \
  int i[kRows];                                    \
  bool in[kRows];                                  \
  _Pragma("unroll") for (int r_ = 0; r_ < kRows; ++r_) { \
    i[r_] = (base) + r_ * (rows).stride + threadIdx.x;   \
    in[r_] = i[r_] < (rows).n;                           \
  }

// Shared prologue: FP32 copy of A (CSR and ELL), FP32 inverse diagonal, b.b
// and the count of zero diagonals; false when the kernel must leave.
template <typename V, bool L1>
__device__ bool prologue(const KrylovArgs& a, const MixedArgsT<V>& m, VGrid& g, Red& R, const Rows& rows, double& bnrm,
                         bool& diag_bad) {
  MGPU_TILES(rows, base) {
    const int i = base + threadIdx.x;
    double c[2] = {0.0, 0.0};
    if (i < rows.n) {
      const int rb = a.row_ptr[i], re = a.row_ptr[i + 1];
      for (int k = rb; k < re; ++k) m.a32[k] = (V)a.aval[k];
      if (m.ell_col)
        for (int t = 0; t < m.ell_w; ++t) m.ell_val[(long)t * m.ell_ld + i] = t < re - rb ? (V)a.aval[rb + t] : V(0);
      if (m.ell64)
        for (int t = 0; t < m.ell_w; ++t) m.ell64[(long)t * m.ell_ld + i] = t < re - rb ? a.aval[rb + t] : 0.0;
      if (a.zero_x) a.x[i] = 0.0;
      const double dg = a.aval[a.diag[i]];
      if (fabs(dg) < DTINY) c[1] = 1.0;
      m.dinv[i] = (V)(1.0 / dg);
      c[0] = a.b[i] * a.b[i];
    }
    red_put<2>(R, rows, base, c);
  }
  double v[2];
  if (!red_total<2, L1>(R, rows, g, a.st, v)) return false;
  bnrm = sqrt(v[0]);
  diag_bad = v[1] != 0.0;
  return true;
}

// r = b - A x in FP64; returns |r| through rnorm
template <bool L1>
__device__ bool true_residual(const KrylovArgs& a, VGrid& g, Red& R, const Rows& rows, double& rnorm) {
  MGPU_TILES(rows, base) {
    const int i = base + threadIdx.x;
    double c[1] = {0.0};
    if (i < rows.n) {
      const double ri = a.b[i] - row_spmv64<L1>(a, a.x, i);
      a.r[i] = ri;
      c[0] = ri * ri;
    }
    red_put<1>(R, rows, base, c);
  }
  double v[1];
  if (!red_total<1, L1>(R, rows, g, a.st, v)) return false;
  rnorm = sqrt(v[0]);
  return true;
}

// x += scale * d, then a barrier (neighbours' x are read next)
template <typename V, bool L1>
__device__ bool update_x(const KrylovArgs& a, VGrid& g, const Rows& rows, const V* d, double scale) {
  for (int i = rows.start + threadIdx.x; i < rows.n; i += rows.stride) a.x[i] = fma(scale, (double)d[i], a.x[i]);
  return vg_sync(g, a.st);
}

// Chebyshev-Jacobi preconditioner z = p(D^-1 A) D^-1 rr of degree k on
// [lmax/ratio, lmax]: k-1 SpMV passes, one barrier each. On entry z0 = d =
// D^-1 rr / theta (written by the caller's pass, followed by a barrier). The
// result lands in zout (z0 or z1, ping-pong); the last pass also sums rr.z and
// rr.rr (r64.z in place of rr.z when the FP64 residual r64 is given),
// reduced before returning.
template <typename V, bool L1, int ELL>
__device__ __forceinline__ bool cheb_apply(const KrylovArgs& a, const MixedArgsT<V>& m, VGrid& g, Red& R,
                                           const Rows& rows, const V* rr, V* dch, V* z0, V* z1,
                                           double lmax, V*& zout, double (&red)[2],
                                           const double* r64 = nullptr) {
  const Sp32<V> S = sp32_of(a, m, rows);
  const double lmin = lmax / m.cheb_ratio;
  const double th = 0.5 * (lmax + lmin), de = 0.5 * (lmax - lmin), sg = th / de;
  double rho0 = 1.0 / sg;
  V* zc = z0;
  V* zn = z1;
  red[0] = red[1] = 0.0;
  for (int j = 1; j < m.cheb_k; ++j) {
    const double rho1 = 1.0 / (2.0 * sg - rho0);
    const V c1 = (V)(rho1 * rho0), c2 = (V)(2.0 * rho1 / de);
    const bool last = (j == m.cheb_k - 1);
    with_width<ELL>(S.w, [&](auto wc) {
    constexpr int WC = decltype(wc)::value;
    MGPU_STEPS(rows, base) {
      MGPU_STEP_ROWS(rows, base, ii, in);
      MGPU_SPLIT_FULL(rows, base, FULL, {
        V az[kRows];
        spmv32_rows<V, L1, ELL, FULL, WC>(S, zc, ii, in, az);
_Pragma("unroll") for (int r = 0; r < kRows; ++r) {
          const int i = ii[r];
          double c[2] = {0.0, 0.0};
          if (FULL || in[r]) {
            const V res = S.dinv[i] * (rr[i] - az[r]);
            const V dn = vfma(c1, dch[i], c2 * res);
            dch[i] = dn;
            const V zi = zc[i] + dn;
            zn[i] = zi;
            if (last) {
              c[0] = r64 ? r64[i] * (double)zi : (double)rr[i] * (double)zi;
              c[1] = (double)rr[i] * (double)rr[i];
            }
          }
          if (last) red_put<2>(R, rows, base + r * rows.stride, c);
        }
      })
    }
    });
    if (last) {
      if (!red_total<2, L1>(R, rows, g, a.st, red)) return false;
    } else if (!vg_sync(g, a.st)) {
      return false;
    }
    V* t = zc;
    zc = zn;
    zn = t;
    rho0 = rho1;
  }
  zout = zc;
  return true;
}

// The SpMV passes of the Krylov loops.

// pnew := z + beta pold and q := A pnew in one pass (pnew := z, q := A z when
// first), q formed directly from z and pold rather than recurred; pnew.q
template <typename V, bool L1, int ELL>
__device__ __forceinline__ void pcg_direct_pass(const KrylovArgs& a, const MixedArgsT<V>& m, const Red& R,
                                                const Rows& rows, const V* z, const V* pold, V* pnew, V* q, V beta,
                                                bool first) {
  const Sp32<V> S = sp32_of(a, m, rows);
  with_width<ELL>(S.w, [&](auto wc) {
  constexpr int WC = decltype(wc)::value;
  MGPU_STEPS(rows, base) {
    MGPU_STEP_ROWS(rows, base, ii, in);
    MGPU_SPLIT_FULL(rows, base, FULL, {
      V aq[kRows];
      spmv32_rows_dir<V, L1, ELL, FULL, WC>(S, z, pold, beta, first, ii, in, aq);
_Pragma("unroll") for (int r = 0; r < kRows; ++r) {
        const int i = ii[r];
        double c[1] = {0.0};
        if (FULL || in[r]) {
          const V pi = first ? z[i] : vfma(beta, pold[i], z[i]);
          pnew[i] = pi;
          q[i] = aq[r];
          c[0] = (double)pi * (double)aq[r];
        }
        red_put<1>(R, rows, base + r * rows.stride, c);
      }
    })
  }
  });
}

// v := A ph; r0.v
template <typename V, bool L1, int ELL>
__device__ __forceinline__ void bicg_v_pass(const KrylovArgs& a, const MixedArgsT<V>& m, const Red& R, const Rows& rows,
                                            const V* ph, const V* r0, V* v) {
  const Sp32<V> S = sp32_of(a, m, rows);
  with_width<ELL>(S.w, [&](auto wc) {
  constexpr int WC = decltype(wc)::value;
  MGPU_STEPS(rows, base) {
    MGPU_STEP_ROWS(rows, base, ii, in);
    MGPU_SPLIT_FULL(rows, base, FULL, {
      V vv[kRows];
      spmv32_rows<V, L1, ELL, FULL, WC>(S, ph, ii, in, vv);
_Pragma("unroll") for (int r = 0; r < kRows; ++r) {
        const int i = ii[r];
        double c[1] = {0.0};
        if (FULL || in[r]) {
          v[i] = vv[r];
          c[0] = (double)r0[i] * (double)vv[r];
        }
        red_put<1>(R, rows, base + r * rows.stride, c);
      }
    })
  }
  });
}

// t := A sh; t.t and t.s
template <typename V, bool L1, int ELL>
__device__ __forceinline__ void bicg_t_pass(const KrylovArgs& a, const MixedArgsT<V>& m, const Red& R, const Rows& rows,
                                            const V* sh, const V* s, V* t) {
  const Sp32<V> S = sp32_of(a, m, rows);
  with_width<ELL>(S.w, [&](auto wc) {
  constexpr int WC = decltype(wc)::value;
  MGPU_STEPS(rows, base) {
    MGPU_STEP_ROWS(rows, base, ii, in);
    MGPU_SPLIT_FULL(rows, base, FULL, {
      V tv[kRows];
      spmv32_rows<V, L1, ELL, FULL, WC>(S, sh, ii, in, tv);
_Pragma("unroll") for (int r = 0; r < kRows; ++r) {
        const int i = ii[r];
        double c[2] = {0.0, 0.0};
        if (FULL || in[r]) {
          t[i] = tv[r];
          c[0] = (double)tv[r] * (double)tv[r];
          c[1] = (double)tv[r] * (double)s[i];
        }
        red_put<2>(R, rows, base + r * rows.stride, c);
      }
    })
  }
  });
}

// ---------------------------------------------------------------------------
// PCG (pressure correction): Jacobi or Chebyshev-Jacobi preconditioned
// ---------------------------------------------------------------------------

// PCG in working precision V on the residual scaled by the fixed factor
// sc = 1 / |b - A x0|, with reliable updates: every iteration adds its step to
// the FP64 solution (x += alpha |r0| p); whenever the recursive residual's norm
// has fallen by rel_delta since the last replacement (rel_delta 0: never), or
// says the solve has converged, an FP64 pass forms r = b - A x and puts sc r
// in its place, keeping p, q and r.z, so the Krylov space survives; the true
// residual decides convergence. The FP64 polynomial form runs it with
// V = double and rel_delta 0 (plain FP64 PCG, b - A x only to confirm). q = A
// p is formed directly every iteration (pcg_direct_pass), not recurred. On
// entry a.r holds b - A x0 and rnorm0 its norm. Barriers: every pass that
// writes x, rr or z ends in a reduction (one grid barrier), which is also the
// barrier before the next SpMV pass.
// After a residual replacement in pcg_reliable: start a new direction when
// the replacement came from convergence of the recursive residual (its check
// failed), or when the recursive residual had drifted by more than 2x.
__device__ __forceinline__ bool rel_delta_restart(double rr_true2, double rr_rec2, bool converged) {
  return converged || rr_true2 > 4.0 * rr_rec2;
}

template <typename V, bool L1, int ELL>
__device__ void pcg_reliable(const KrylovArgs& a, const MixedArgsT<V>& m, VGrid& g, Red& R, const Rows& rows,
                             double bnrm, double rnorm0, double lmax, V inv_th) {
  const int n = a.n;
  const V* __restrict__ dinv = m.dinv;
  V *rr = m.w32, *zA = m.w32 + n, *p = m.w32 + 2l * n, *q = m.w32 + 3l * n;
  V *dch = m.w32 + 5l * n, *zB = m.w32 + 6l * n, *pn = m.w32 + 7l * n;  // p double-buffered
  const bool cheb = m.cheb_k > 1;
  const double sc = 1.0 / rnorm0;
  const double stop = a.tol * bnrm * sc;  // |rr| at which the estimate reaches tol
  const double stop2 = stop * stop, delta2 = m.rel_delta * m.rel_delta;
  // rr := sc r, z0 (Jacobi: z = D^-1 rr; Chebyshev: its first term), rr.z
  MGPU_TILES(rows, base) {
    const int i = base + threadIdx.x;
    double c[1] = {0.0};
    if (i < rows.n) {
      const V ri = (V)(ldv(&a.r[i]) * sc);
      rr[i] = ri;
      const V zi = cheb ? dinv[i] * ri * inv_th : dinv[i] * ri;
      if (cheb) dch[i] = zi;
      zA[i] = zi;
      c[0] = (double)ri * (double)zi;
    }
    red_put<1>(R, rows, base, c);
  }
  double t1[1];
  if (!red_total<1, L1>(R, rows, g, a.st, t1)) return;
  double rzn = t1[0], rz = 0.0, rr_ref = 1.0, rnorm = rnorm0;
  int total = 0, ierr = 0;
  bool first = true;
  while (true) {
    V* z = zA;
    if (cheb) {
      double red[2];  // (rr.z, rr.rr)
      if (!cheb_apply<V, L1, ELL>(a, m, g, R, rows, rr, dch, zA, zB, lmax, z, red)) return;
      rzn = red[0];
    }
    V beta = V(0);
    if (!first) {
      if (fabs(rz) < DTINY) {
        ierr = 2;
        break;
      }
      beta = (V)(rzn / rz);
    }
    rz = rzn;
    ++total;
    pcg_direct_pass<V, L1, ELL>(a, m, R, rows, z, p, pn, q, beta, first);
    {
      V* t = p;
      p = pn;
      pn = t;
    }
    first = false;
    double pq[1];
    if (!red_total<1, L1>(R, rows, g, a.st, pq)) return;
    if (fabs(pq[0]) < DTINY) {
      ierr = 2;
      break;
    }
    const double al = rz / pq[0];
    const V af = (V)al;
    const double ax = al * rnorm0;  // the step in unscaled units
    // x += ax p (FP64), rr -= af q, z0; sums rr.rr and rr.z
    MGPU_TILES(rows, base) {
      const int i = base + threadIdx.x;
      double c[2] = {0.0, 0.0};
      if (i < rows.n) {
        a.x[i] = fma(ax, (double)p[i], a.x[i]);
        const V ri = vfma(-af, q[i], rr[i]);
        rr[i] = ri;
        const V zi = cheb ? dinv[i] * ri * inv_th : dinv[i] * ri;
        if (cheb) dch[i] = zi;
        zA[i] = zi;
        c[0] = (double)ri * (double)ri;
        c[1] = (double)ri * (double)zi;
      }
      red_put<2>(R, rows, base, c);
    }
    double s2[2];
    if (!red_total<2, L1>(R, rows, g, a.st, s2)) return;
    rzn = s2[1];
    if (!(s2[0] <= stop2 || s2[0] <= delta2 * rr_ref || total >= a.maxit)) continue;
    const double rec2 = s2[0];  // the recursive residual's rr.rr before the replacement
    // replacement: r = b - A x in FP64, rr := sc r, z0; sums r.r and rr.z
    MGPU_TILES(rows, base) {
      const int i = base + threadIdx.x;
      double c[2] = {0.0, 0.0};
      if (i < rows.n) {
        const double ri = a.b[i] - row_spmv64<L1>(a, a.x, i);
        const V rf = (V)(ri * sc);
        rr[i] = rf;
        const V zi = cheb ? dinv[i] * rf * inv_th : dinv[i] * rf;
        if (cheb) dch[i] = zi;
        zA[i] = zi;
        c[0] = ri * ri;
        c[1] = (double)rf * (double)zi;
      }
      red_put<2>(R, rows, base, c);
    }
    double t2[2];
    if (!red_total<2, L1>(R, rows, g, a.st, t2)) return;
    rnorm = sqrt(t2[0]);
    const double res = rnorm / bnrm;
    if (res <= a.tol) {
      write_result_m(a, g, total, res, 0);
      return;
    }
    if (total >= a.maxit) {
      ierr = 1;
      break;
    }
    rr_ref = (rnorm * sc) * (rnorm * sc);
    rzn = t2[1];
    // the recursive residual reached the tolerance (or, with rel_delta > 0,
    // fell by delta) while the true one did not: the kept direction belongs to
    // the drifted residual. A restart from the true residual (beta = 0) keeps
    // a solve at its attainable accuracy stagnating instead of diverging; the
    // FP64 polynomial form at lin_tol 1e-12 and degree 24 diverged on the
    // channel's second pressure system when the direction was kept up to a
    // drift of 2x.
    if (rel_delta_restart(rr_ref, rec2, s2[0] <= stop2)) first = true;
  }
  write_result_m(a, g, total, rnorm / bnrm, ierr);
}

// ---------------------------------------------------------------------------
// The mixed form's PCG: FP64 conjugate gradients, FP32 polynomial
// ---------------------------------------------------------------------------

// y = A (z + beta pold) in FP64 from the FP64 ELL values (the CSR values
// without an ELL copy), each gathered entry formed as its owner row forms its
// new direction (first: y = A z): pold FP64, z the FP32 preconditioned
// residual.
template <bool L1, int ELL, bool FULL, int WC = 0>
__device__ __forceinline__ void spmv64_rows_dir(const Sp32<float>& S, const double* __restrict__ ev,
                                                const KrylovArgs& a, const float* z, const double* pold, double beta,
                                                bool first, const int (&i)[kRows], const bool (&in0)[kRows],
                                                double (&y)[kRows]) {
  bool in[kRows];
#pragma unroll
  for (int r = 0; r < kRows; ++r) in[r] = FULL || in0[r];
  if constexpr (ELL) {
    constexpr int WMAX = WC ? WC : 8;  // WC: the ELL width known at compile time
    const int W = WC ? WC : S.w;
    double v[kRows][WMAX], xv[kRows][WMAX];
    int c[kRows][WMAX];
#pragma unroll
    for (int r = 0; r < kRows; ++r)
#pragma unroll
      for (int t = 0; t < WMAX; ++t)
        if (t < W && in[r]) {
          c[r][t] = S.ecol[t * S.ld + i[r]];
          v[r][t] = ev[t * S.ld + i[r]];
        }
    if constexpr (ELL == 2) {
#pragma unroll
      for (int r = 0; r < kRows; ++r) {
        const int j = i[r] + S.pf;
        if (j < S.n) {
#pragma unroll
          for (int t = 0; t < WMAX; ++t)
            if (t < W) {
              prefetch_l2(S.ecol + t * S.ld + j);
              prefetch_l2(ev + t * S.ld + j);
            }
        }
      }
    }
#pragma unroll
    for (int r = 0; r < kRows; ++r)
#pragma unroll
      for (int t = 0; t < WMAX; ++t)
        if (t < W && in[r])
          xv[r][t] = first ? (double)ldv(&z[c[r][t]]) : fma(beta, ldv(&pold[c[r][t]]), (double)ldv(&z[c[r][t]]));
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      double acc = 0.0;
#pragma unroll
      for (int t = 0; t < WMAX; ++t)
        if (t < W && in[r]) acc = fma(v[r][t], xv[r][t], acc);
      y[r] = acc;
    }
  } else {
#pragma unroll
    for (int r = 0; r < kRows; ++r) {
      double acc = 0.0;
      if (in[r]) {
        const int e = a.row_ptr[i[r] + 1];
        for (int k = a.row_ptr[i[r]]; k < e; ++k) {
          const int cc = a.col[k];
          const double x = first ? (double)ldv(&z[cc]) : fma(beta, ldv(&pold[cc]), (double)ldv(&z[cc]));
          acc = fma(a.aval[k], x, acc);
        }
      }
      y[r] = acc;
    }
  }
}

// pnew := z + beta pold and q := A pnew (FP64) in one pass; pnew.q
template <bool L1, int ELL>
__device__ __forceinline__ void pcg_hybrid_direct_pass(const KrylovArgs& a, const MixedArgs& m, const Red& R,
                                                       const Rows& rows, const float* z, const double* pold,
                                                       double* pnew, double* q, double beta, bool first) {
  const Sp32<float> S = sp32_of(a, m, rows);
  const double* __restrict__ ev = m.ell64;
  with_width<ELL>(S.w, [&](auto wc) {
  constexpr int WC = decltype(wc)::value;
  MGPU_STEPS(rows, base) {
    MGPU_STEP_ROWS(rows, base, ii, in);
    MGPU_SPLIT_FULL(rows, base, FULL, {
      double aq[kRows];
      spmv64_rows_dir<L1, ELL, FULL, WC>(S, ev, a, z, pold, beta, first, ii, in, aq);
_Pragma("unroll") for (int r = 0; r < kRows; ++r) {
        const int i = ii[r];
        double c[1] = {0.0};
        if (FULL || in[r]) {
          const double pi = first ? (double)z[i] : fma(beta, pold[i], (double)z[i]);
          pnew[i] = pi;
          q[i] = aq[r];
          c[0] = pi * aq[r];
        }
        red_put<1>(R, rows, base + r * rows.stride, c);
      }
    })
  }
  });
}

// PCG in FP64 (x, the residual, the search direction and q = A p, every sum)
// with the preconditioner in FP32: the Chebyshev-Jacobi polynomial runs on an
// FP32 copy of the residual with the FP32 matrix copy and FP32 vectors. The
// polynomial's passes are 15 of the 17 passes of an iteration at degree 16,
// so the iteration moves nearly the FP32 form's bytes, while the conjugate
// gradient recurrence keeps the FP64 form's convergence (a CG stream run in
// FP32 loses it: 71 against 52 iterations on the 524k channel's pressure
// systems). The residual is carried scaled by sc = 1 / |b - A x0|. When it
// says the solve has converged, an FP64 pass forms b - A x and decides; if
// that is still above the tolerance the iteration restarts from it. On entry
// a.r holds b - A x0 and rnorm0 its norm. Every pass that writes what the
// next pass gathers ends in a reduction (one grid barrier).
template <bool L1, int ELL>
__device__ void pcg_hybrid(const KrylovArgs& a, const MixedArgs& m, VGrid& g, Red& R, const Rows& rows, double bnrm,
                           double rnorm0, double lmax, float inv_th) {
  const int n = a.n;
  const float* __restrict__ dinv = m.dinv;
  float *rr = m.w32, *zA = m.w32 + n, *dch = m.w32 + 5l * n, *zB = m.w32 + 6l * n;
  double *rs = a.r, *p = a.p, *pn = a.s, *q = a.v;  // p double-buffered
  const bool cheb = m.cheb_k > 1;
  const double sc = 1.0 / rnorm0;
  const double stop = a.tol * bnrm * sc;  // |rs| at which the solve has converged
  const double stop2 = stop * stop;
  // rs := sc r, its FP32 copy, z0 (Jacobi: z = D^-1 rr; Chebyshev: its first
  // term); rs.z0
  MGPU_TILES(rows, base) {
    const int i = base + threadIdx.x;
    double c[1] = {0.0};
    if (i < rows.n) {
      const double ri = ldv(&a.r[i]) * sc;
      rs[i] = ri;
      const float rf = (float)ri;
      rr[i] = rf;
      const float zi = cheb ? dinv[i] * rf * inv_th : dinv[i] * rf;
      if (cheb) dch[i] = zi;
      zA[i] = zi;
      c[0] = ri * (double)zi;
    }
    red_put<1>(R, rows, base, c);
  }
  double t1[1];
  if (!red_total<1, L1>(R, rows, g, a.st, t1)) return;
  double rzn = t1[0], rz = 0.0, rnorm = rnorm0;
  int total = 0, ierr = 0;
  bool first = true;
  while (true) {
    float* z = zA;
    if (cheb) {
      double red[2];  // (rs.z, rr.rr)
      if (!cheb_apply<float, L1, ELL>(a, m, g, R, rows, rr, dch, zA, zB, lmax, z, red, rs)) return;
      rzn = red[0];
    }
    double beta = 0.0;
    if (!first) {
      if (fabs(rz) < DTINY) {
        ierr = 2;
        break;
      }
      beta = rzn / rz;
    }
    rz = rzn;
    ++total;
    pcg_hybrid_direct_pass<L1, ELL>(a, m, R, rows, z, p, pn, q, beta, first);
    {
      double* t = p;
      p = pn;
      pn = t;
    }
    first = false;
    double pq[1];
    if (!red_total<1, L1>(R, rows, g, a.st, pq)) return;
    if (fabs(pq[0]) < DTINY) {
      ierr = 2;
      break;
    }
    const double al = rz / pq[0];
    const double ax = al * rnorm0;  // the step in unscaled units
    // x += ax p, rs -= al q, FP32 copy and z0; sums rs.rs and rs.z0
    MGPU_TILES(rows, base) {
      const int i = base + threadIdx.x;
      double c[2] = {0.0, 0.0};
      if (i < rows.n) {
        a.x[i] = fma(ax, p[i], a.x[i]);
        const double ri = fma(-al, q[i], rs[i]);
        rs[i] = ri;
        const float rf = (float)ri;
        rr[i] = rf;
        const float zi = cheb ? dinv[i] * rf * inv_th : dinv[i] * rf;
        if (cheb) dch[i] = zi;
        zA[i] = zi;
        c[0] = ri * ri;
        c[1] = ri * (double)zi;
      }
      red_put<2>(R, rows, base, c);
    }
    double s2[2];
    if (!red_total<2, L1>(R, rows, g, a.st, s2)) return;
    rzn = s2[1];
    if (!(s2[0] <= stop2 || total >= a.maxit)) continue;
    // r = b - A x in FP64 decides; rs := sc r, FP32 copy, z0; sums r.r, rs.z0
    MGPU_TILES(rows, base) {
      const int i = base + threadIdx.x;
      double c[2] = {0.0, 0.0};
      if (i < rows.n) {
        const double ri = a.b[i] - row_spmv64<L1>(a, a.x, i);
        const double si = ri * sc;
        rs[i] = si;
        const float rf = (float)si;
        rr[i] = rf;
        const float zi = cheb ? dinv[i] * rf * inv_th : dinv[i] * rf;
        if (cheb) dch[i] = zi;
        zA[i] = zi;
        c[0] = ri * ri;
        c[1] = si * (double)zi;
      }
      red_put<2>(R, rows, base, c);
    }
    double t2[2];
    if (!red_total<2, L1>(R, rows, g, a.st, t2)) return;
    rnorm = sqrt(t2[0]);
    const double res = rnorm / bnrm;
    if (res <= a.tol) {
      write_result_m(a, g, total, res, 0);
      return;
    }
    if (total >= a.maxit) {
      ierr = 1;
      break;
    }
    rzn = t2[1];
    first = true;  // the recursive residual had drifted: restart from the true one
  }
  write_result_m(a, g, total, rnorm / bnrm, ierr);
}

template <typename V, bool L1, int ELL, bool DYN = false>
__device__ void pcg_mixed_body(const KrylovArgs& a, const MixedArgsT<V>& m, VGrid& g) {
  if (a.st->abort) return;
  const int n = a.n;
  if (!fits_group(n, g) || (DYN && !fits_slots(n, g, m.cp_slots))) {
    // unreachable through the launchers: reported as a breakdown
    write_result_m(a, g, 0, 0.0, 2);
    return;
  }
  const Rows rows = block_rows(n, g);
  Red R = make_red<V, DYN>(m, n);
  const bool cheb = m.cheb_k > 1;
  double bnrm;
  bool diag_bad;
  if (!prologue<V, L1>(a, m, g, R, rows, bnrm, diag_bad)) return;
  if (bnrm == 0.0) {
    for (int i = rows.start + threadIdx.x; i < rows.n; i += rows.stride) a.x[i] = 0.0;
    write_result_m(a, g, 0, 0.0, 0);
    return;
  }
  if (diag_bad) {
    write_result_m(a, g, 0, 0.0, 2);
    return;
  }
  // Chebyshev interval: Gershgorin bound of D^-1 A (row sum of |a_ij| / a_ii);
  // a maximum is exact in any order
  double lmax = 2.0, th = 1.0;
  if (cheb) {
    double gm = 0.0;
    for (int i = rows.start + threadIdx.x; i < rows.n; i += rows.stride) {
      double s = 0.0;
      for (int k = a.row_ptr[i]; k < a.row_ptr[i + 1]; ++k) s += fabs(a.aval[k]);
      gm = fmax(gm, s / fabs(a.aval[a.diag[i]]));
    }
    if (!vg_max<L1>(gm, g, a.st)) return;
    lmax = gm;
    th = 0.5 * (lmax + lmax / m.cheb_ratio);
  }
  const V inv_th = (V)(1.0 / th);
  double rnorm;
  if (!true_residual<L1>(a, g, R, rows, rnorm)) return;
  double res = rnorm / bnrm;
  if (res <= a.tol) {
    write_result_m(a, g, 0, res, 0);
    return;
  }
  if constexpr (sizeof(V) == 4)
    pcg_hybrid<L1, ELL>(a, m, g, R, rows, bnrm, rnorm, lmax, inv_th);
  else
    pcg_reliable<V, L1, ELL>(a, m, g, R, rows, bnrm, rnorm, lmax, inv_th);
}

// ---------------------------------------------------------------------------
// BiCGStab (momentum): right Jacobi preconditioning
// ---------------------------------------------------------------------------
template <typename V, bool L1, int ELL, bool DYN = false>
__device__ void bicgstab_mixed_body(const KrylovArgs& a, const MixedArgsT<V>& m, VGrid& g) {
  if (a.st->abort) return;
  const int n = a.n;
  if (!fits_group(n, g) || (DYN && !fits_slots(n, g, m.cp_slots))) {
    // unreachable through the launchers: reported as a breakdown
    write_result_m(a, g, 0, 0.0, 2);
    return;
  }
  const Rows rows = block_rows(n, g);
  const V* __restrict__ dinv = m.dinv;
  Red R = make_red<V, DYN>(m, n);
  V* W = m.w32;
  V *r = W, *r0 = W + n, *p = W + 2l * n, *v = W + 3l * n, *s = W + 4l * n, *t = W + 5l * n,
        *ph = W + 6l * n, *sh = W + 7l * n, *d = W + 8l * n;
  double bnrm;
  bool diag_bad;
  if (!prologue<V, L1>(a, m, g, R, rows, bnrm, diag_bad)) return;
  if (bnrm == 0.0) {
    for (int i = rows.start + threadIdx.x; i < rows.n; i += rows.stride) a.x[i] = 0.0;
    write_result_m(a, g, 0, 0.0, 0);
    return;
  }
  if (diag_bad) {
    write_result_m(a, g, 0, 0.0, 12);
    return;
  }
  double rnorm;
  if (!true_residual<L1>(a, g, R, rows, rnorm)) return;
  double res = rnorm / bnrm;
  if (res <= a.tol) {
    write_result_m(a, g, 0, res, 0);
    return;
  }
  int total = 0, ierr = 0;
  while (true) {
    const double inv = 1.0 / rnorm;
    MGPU_TILES(rows, base) {
      const int i = base + threadIdx.x;
      double c[1] = {0.0};
      if (i < rows.n) {
        const V ri = (V)(ldv(&a.r[i]) * inv);
        r[i] = ri;
        r0[i] = ri;
        p[i] = V(0);
        v[i] = V(0);
        d[i] = V(0);
        c[0] = (double)ri * (double)ri;
      }
      red_put<1>(R, rows, base, c);
    }
    double w1[1];
    if (!red_total<1, L1>(R, rows, g, a.st, w1)) return;
    // FP32 inner solves gain tau per refinement step; in FP64 the inner solve
    // goes straight to the tolerance on the (scaled) residual
    const double tau = sizeof(V) == sizeof(double) ? a.tol * bnrm / rnorm : m.tau;
    const double target = tau * tau * w1[0];
    double rho_next = w1[0], rho_old = 1.0, alpha = 1.0, omega = 1.0;
    while (true) {
      ++total;
      const double rho = rho_next;
      if (fabs(rho) < DTINY) {
        ierr = 2;
        break;
      }
      const V beta = (V)((rho / rho_old) * (alpha / omega));
      const V om = (V)omega;
      for (int i = rows.start + threadIdx.x; i < rows.n; i += rows.stride) {
        const V pi = vfma(beta, vfma(-om, v[i], p[i]), r[i]);
        p[i] = pi;
        ph[i] = dinv[i] * pi;
      }
      if (!vg_sync(g, a.st)) return;
      bicg_v_pass<V, L1, ELL>(a, m, R, rows, ph, r0, v);
      double d1[1];
      if (!red_total<1, L1>(R, rows, g, a.st, d1)) return;
      alpha = rho / d1[0];
      const V af = (V)alpha;
      MGPU_TILES(rows, base) {
        const int i = base + threadIdx.x;
        double c[1] = {0.0};
        if (i < rows.n) {
          const V si = vfma(-af, v[i], r[i]);
          s[i] = si;
          sh[i] = dinv[i] * si;
          c[0] = (double)si * (double)si;
        }
        red_put<1>(R, rows, base, c);
      }
      double d2[1];
      if (!red_total<1, L1>(R, rows, g, a.st, d2)) return;
      if (d2[0] <= target || total >= a.maxit) {
        for (int i = rows.start + threadIdx.x; i < rows.n; i += rows.stride) d[i] = vfma(af, ph[i], d[i]);
        break;
      }
      bicg_t_pass<V, L1, ELL>(a, m, R, rows, sh, s, t);
      double d3[2];
      if (!red_total<2, L1>(R, rows, g, a.st, d3)) return;
      if (d3[0] < DTINY) {
        ierr = 2;
        break;
      }
      omega = d3[1] / d3[0];
      if (fabs(omega) < DTINY) {
        ierr = 2;
        break;
      }
      const V omf = (V)omega;
      MGPU_TILES(rows, base) {
        const int i = base + threadIdx.x;
        double c[2] = {0.0, 0.0};
        if (i < rows.n) {
          d[i] = vfma(omf, sh[i], vfma(af, ph[i], d[i]));
          const V ri = vfma(-omf, t[i], s[i]);
          r[i] = ri;
          c[0] = (double)ri * (double)ri;
          c[1] = (double)ri * (double)r0[i];
        }
        red_put<2>(R, rows, base, c);
      }
      double d4[2];
      if (!red_total<2, L1>(R, rows, g, a.st, d4)) return;
      if (d4[0] <= target || total >= a.maxit) break;
      rho_next = d4[1];
      rho_old = rho;
    }
    if (ierr == 2) break;
    if (!update_x<V, L1>(a, g, rows, d, rnorm)) return;
    if (!true_residual<L1>(a, g, R, rows, rnorm)) return;
    res = rnorm / bnrm;
    if (res <= a.tol) {
      write_result_m(a, g, total, res, 0);
      return;
    }
    if (total >= a.maxit) {
      ierr = 1;
      break;
    }
  }
  write_result_m(a, g, total, res, ierr);
}

#undef MGPU_TILES
#undef MGPU_STEPS
#undef MGPU_STEP_ROWS
#undef MGPU_SPLIT_FULL

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

// One solve as a cooperative launch: fn1 for a single block, fnN for a grid.
template <typename V>
int launch_mixed(const void* fn1, const void* fnN, const KrylovArgs& a, const MixedArgsT<V>& m, cudaStream_t s) {
  if (a.n > kMixedMaxRows || !m.red) {
    set_error("mixed-precision solve: system larger than 2^24 rows or no reduction work space");
    return MGPU_E_ARG;
  }
  // one 512-thread block up to the single-block threshold (and the rows one
  // block may hold), else the kernel's co-resident grid at ~2 rows per thread
  int block = 0;
  int grid = krylov_grid(a.n, block, 0);
  if (grid == 1 && a.n > kBlockMaxRows) grid = 2;
  // grid kernels: dynamic shared memory for the block's chunk sums (2 sums x
  // 8 chunks per tile of 256 rows, for the most tiles a block owns)
  int dyn = 0, cps = 0;
  if (grid > 1) {
    block = 256;
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fnN, block, (size_t)16 * kBlockMaxChunks);
    if (per < 1) per = 1;
    const long want = ((long)a.n + 2l * block - 1) / (2l * block);
    grid = (int)std::min<long>(std::max<long>(want, 2), (long)sms * per);
    const long rows_per_block = ((long)a.n + grid - 1) / grid;
    cps = (int)std::min<long>((rows_per_block + block - 1) / block * (block / 32), kBlockMaxChunks);
    dyn = 16 * cps;
  }
  if ((long)grid * kBlockMaxRows < a.n) {
    set_error("mixed-precision solve: too many rows per block for the co-resident grid");
    return MGPU_E_ARG;
  }
  KrylovArgs aa = a;
  MixedArgsT<V> mm = m;
  mm.cp_slots = cps;
  void* args[] = {&aa, &mm};
  cudaError_t e = cudaMemsetAsync(a.bar, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return cuda_fail(e, "barrier reset", __FILE__, __LINE__);
  e = cudaLaunchCooperativeKernel(grid == 1 ? fn1 : fnN, dim3(grid), dim3(block), args, (size_t)dyn, s);
  if (e != cudaSuccess) return cuda_fail(e, "cooperative launch (mixed)", __FILE__, __LINE__);
  return 0;
}

// A single-case solve's kernels: ELL (prefetching when the system is larger
// than the L2 share, m.pf) or CSR; one block runs without the prefetch.
template <typename V>
int ell_mode(const MixedArgsT<V>& m) { return m.ell_col ? (m.pf ? 2 : 1) : 0; }

}  // namespace
}  // namespace mgpu
