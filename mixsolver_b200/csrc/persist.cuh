// persist.cuh -- primitives of the persistent (cooperative) Krylov kernels:
// bounded grid barrier, deterministic grid-wide sums, vector loads.
#pragma once

#include "case.cuh"

namespace mgpu {
namespace {

constexpr unsigned kSpinLimit = 1u << 25;  // ~2 s of polling: then flag a timeout

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_acquire_i32(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// A group of co-resident blocks working on one system: the whole grid of a
// single-system launch, or one system's share of a batched launch.
struct VGrid {
  int nb;    // blocks in the group
  int rank;  // this block's rank in the group
  unsigned long long* bar;  // the group's barrier counter
  double* partials;         // the group's reduction partials (2 halves of 4 * nb)
  int half;                 // half of the partials the next reduction writes
  // The counter value that opens this block's next barrier, when every
  // barrier on the counter since it was zeroed went through this object (all
  // blocks then take the same barriers in the same order); 0 when unknown,
  // derived from the arrival's returned count instead.
  unsigned long long next;
  __device__ int gtid() const { return rank * blockDim.x + threadIdx.x; }
  __device__ int gstr() const { return nb * blockDim.x; }
  // Consecutive reductions alternate between the two halves: a block that
  // leaves reduction k early and writes its share of k+1 cannot overwrite a
  // partial of k that a slower block is still reading, because every block
  // reads k's partials before it arrives at k+1's barrier, and k+2 (the next
  // user of the same half) writes only after that barrier.
  __device__ double* next_partials() {
    double* p = partials + (half ? 4 * nb : 0);
    half ^= 1;
    return p;
  }
};

// counted: the counter was zeroed for this launch and every barrier of the
// kernel goes through the returned object (VGrid::next).
__device__ __forceinline__ VGrid whole_grid(unsigned long long* bar, double* partials, bool counted = false) {
  return VGrid{(int)gridDim.x, (int)blockIdx.x, bar, partials, 0, counted ? (unsigned long long)gridDim.x : 0ull};
}

// Bounded barrier of a group over a monotone 64-bit arrival counter (zeroed
// before every launch; all blocks of the group are co-resident). Each block
// adds one arrival and waits until the counter reaches the end of the current
// round. While it waits it looks at the status every 4096 polls: once any
// block has flagged a timeout (st may be null: no status) the wait ends. A
// wait that runs out flags the timeout. Returns false in both cases; the
// caller then leaves the kernel. The status may lower the limit on failed
// polls (DevStatus::spin_limit, from the spin_limit tuning key; 1 gives up at
// the first poll that finds the barrier open) so that a test can make a wait
// run out on purpose.
// Ordering: __syncthreads puts the block's writes before thread 0's arrival,
// a release at GPU scope; thread 0's polls are acquires, and the closing
// __syncthreads puts them before the block's later loads. Release and acquire
// are cumulative in the PTX memory model, so every block's pre-barrier writes
// are visible to every block after it without a separate fence.
// With g.next known the arrival is a reduction whose result nobody waits for
// (red.release) and the barrier opens at g.next; otherwise the arrival
// returns the count and the barrier opens at the end of its round.
__device__ bool vg_sync(VGrid& g, DevStatus* st) {
  __shared__ int s_ok;
  if (g.nb == 1) {
    __syncthreads();
    return true;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    unsigned long long* bar = g.bar;
    const unsigned long long nb = g.nb;
    unsigned long long target;
    if (g.next) {
      asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(bar) : "memory");
      target = g.next;
    } else {
      unsigned long long old;
      asm volatile("atom.add.release.gpu.global.u64 %0, [%1], 1;" : "=l"(old) : "l"(bar) : "memory");
      target = (old / nb + 1ull) * nb;
    }
    const unsigned pns = st ? st->poll_ns : 0u;
    // the built-in bound counts polls of ~60 ns; a back-off stretches each
    const unsigned limit = (st && st->spin_limit)
                               ? st->spin_limit
                               : (unsigned)((unsigned long long)kSpinLimit * 64ull / (64ull + pns));
    unsigned spins = 0;
    while (ld_acquire_u64(bar) < target) {
      ++spins;
      if (pns)
        __nanosleep(pns);
      else if (spins > 256u)
        __nanosleep(64);
      if ((spins & 4095u) == 0 && st && ld_acquire_i32(&st->timeout) != 0) {
        ok = 0;
        break;
      }
      if (spins >= limit) {
        if (st) atomicExch(&st->timeout, 1);
        ok = 0;
        break;
      }
    }
    s_ok = ok;
  }
  if (g.next) g.next += (unsigned long long)g.nb;
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ bool grid_sync(unsigned long long* bar, DevStatus* st) {
  VGrid g{(int)gridDim.x, (int)blockIdx.x, bar, nullptr, 0, 0ull};
  return vg_sync(g, st);
}

// Vector loads inside a persistent kernel. A block reads data that other
// blocks wrote only after a grid barrier (vg_sync), whose acquire load and
// GPU-scope fence follow the other blocks' fence + arrival: by the PTX memory
// model those writes then precede every later load of the block (the pattern
// of a cooperative grid sync), so plain loads, which may hit in L1, are
// coherent with one block or many.
template <typename T>
__device__ __forceinline__ T ldv(const T* p) {
  return *p;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = v + __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Deterministic grid-wide sum of NQ values: block tree -> per-block partials
// -> barrier -> every block sums the partials in the same fixed order (each
// thread a strided share, then the same block tree), so all blocks hold the
// identical total. The partials are fetched by all threads at once: a single
// L2 round trip instead of a serial chain.
template <int NQ, bool L1>
__device__ bool vg_sum(double (&v)[NQ], VGrid& g, DevStatus* st) {
  static_assert(NQ <= 4, "at most 4 sums per reduction");
  double* partials = g.nb == 1 ? nullptr : g.next_partials();
  __shared__ double sh[NQ][32];
  __shared__ double tot[NQ];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double s = warp_sum(v[q]);
    if (lane == 0) sh[q][warp] = s;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double s = lane < nw ? sh[q][lane] : 0.0;
      s = warp_sum(s);
      if (lane == 0) {
        if (g.nb == 1)
          tot[q] = s;
        else
          partials[q * g.nb + g.rank] = s;
      }
    }
  }
  if (g.nb == 1) {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NQ; ++q) v[q] = tot[q];
    __syncthreads();
    return true;
  }
  if (!vg_sync(g, st)) return false;
  const int G = g.nb;
  double w[NQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) {
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
    const int j0 = threadIdx.x, B = blockDim.x;
    if (j0 < G) t0 = ldv(&partials[q * G + j0]);
    if (j0 + B < G) t1 = ldv(&partials[q * G + j0 + B]);
    if (j0 + 2 * B < G) t2 = ldv(&partials[q * G + j0 + 2 * B]);
    if (j0 + 3 * B < G) t3 = ldv(&partials[q * G + j0 + 3 * B]);
    double s = ((t0 + t1) + t2) + t3;
    for (int j = j0 + 4 * B; j < G; j += B) s = s + ldv(&partials[q * G + j]);
    w[q] = warp_sum(s);
  }
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NQ; ++q) sh[q][warp] = w[q];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      double s = lane < nw ? sh[q][lane] : 0.0;
      s = warp_sum(s);
      if (lane == 0) tot[q] = s;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < NQ; ++q) v[q] = tot[q];
  __syncthreads();
  return true;
}

// Grid-wide maximum of one non-negative value (exact, order-independent).
template <bool L1>
__device__ bool vg_max(double& v, VGrid& g, DevStatus* st) {
  double* partials = g.nb == 1 ? nullptr : g.next_partials();
  __shared__ double sh[32];
  __shared__ double tot;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double m = v;
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) sh[warp] = m;
  __syncthreads();
  if (warp == 0) {
    double s = lane < nw ? sh[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
    if (lane == 0) {
      if (g.nb == 1)
        tot = s;
      else
        partials[g.rank] = s;
    }
  }
  if (g.nb > 1) {
    if (!vg_sync(g, st)) return false;
    double s = 0.0;
    for (int j = threadIdx.x; j < g.nb; j += blockDim.x) s = fmax(s, ldv(&partials[j]));
    for (int o = 16; o > 0; o >>= 1) s = fmax(s, __shfl_xor_sync(0xffffffffu, s, o));
    __syncthreads();
    if (lane == 0) sh[warp] = s;
    __syncthreads();
    if (warp == 0) {
      double t = lane < nw ? sh[lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) t = fmax(t, __shfl_xor_sync(0xffffffffu, t, o));
      if (lane == 0) tot = t;
    }
  }
  __syncthreads();
  v = tot;
  __syncthreads();
  return true;
}

}  // namespace
}  // namespace mgpu
