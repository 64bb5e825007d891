// krylov_mixed.cu -- kernels and launchers of the mixed-precision form: FP32
// inner Krylov solves inside FP64 refinement (the bodies, shared with the FP64
// polynomial form, are in krylov_poly.cuh), one cooperative launch per solve,
// and the batched lane kernel that runs many systems in one launch.

#include <algorithm>
#include <type_traits>

#include "krylov_poly.cuh"

namespace mgpu {
extern int g_mixed_occ;  // krylov.cu: the mixed_blocks_per_sm tuning key
extern int g_batch_occ;  // krylov.cu: the batch_blocks_per_sm tuning key
namespace {

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------

// OCC: resident blocks per SM the register budget is sized for (2: 128
// registers a thread; 3: 80; 4: 64; 5: 48), chosen at launch for both solvers
// (tuning key "mixed_blocks_per_sm")
template <bool L1, int ELL, int OCC = 2>
__global__ void __launch_bounds__(L1 ? 512 : 256, L1 ? 1 : OCC) k_pcg_mixed(KrylovArgs a, MixedArgs m) {
  VGrid g = whole_grid(a.bar, a.partials, true);
  pcg_mixed_body<float, L1, ELL, !L1>(a, m, g);
}

template <bool L1, int ELL, int OCC = 2>
__global__ void __launch_bounds__(L1 ? 512 : 256, L1 ? 1 : OCC) k_bicgstab_mixed(KrylovArgs a, MixedArgs m) {
  VGrid g = whole_grid(a.bar, a.partials, true);
  bicgstab_mixed_body<float, L1, ELL, !L1>(a, m, g);
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

// Next system of a lane: its own class queue first, then narrower classes.
__device__ __forceinline__ int lane_fetch(const LanePlan& p, int cls) {
  for (int c = cls; c < p.ncls; ++c) {
    const int k = atomicAdd(&p.q_head[c], 1);
    if (k < p.q_start[c + 1] - p.q_start[c]) return p.q_items[p.q_start[c] + k];
  }
  return -1;
}

// Batched solves. The launch is split into lanes; a lane is a group of
// co-resident blocks with its own barrier counter and max partials. Its first
// block takes the lane's next system from the class queues and publishes it
// in a lane slot (two slots, alternating, so a block still reading one slot
// is never overwritten); the lane barrier makes it visible to the lane's
// other blocks. Every lane runs the multi-block body (a lane of one block
// synchronises with __syncthreads): one body per kernel, inlined, with
// the system's descriptor read through a read-only pointer, keeps the
// descriptor fields out of the register budget.
template <bool PCG, int ELL, int OCC = 2>
__global__ void __launch_bounds__(256, OCC) k_mixed_batch(LanePlan p) {
  __shared__ int s_idx;
  const int li = p.block_lane[blockIdx.x];
  const BatchLane L = p.lanes[li];
  VGrid g{L.nblocks, (int)blockIdx.x - L.first_block, p.bars + li, p.partials + 8l * L.first_block, 0,
          (unsigned long long)L.nblocks};  // lane counters are zeroed before the launch
  if (p.lane_t && g.rank == 0 && threadIdx.x == 0) p.lane_t[2 * li] = globaltimer_ns();
  for (int j = 0;; ++j) {
    __syncthreads();  // every thread is done with the previous system
    if (threadIdx.x == 0) {
      if (g.nb == 1)
        s_idx = lane_fetch(p, L.cls);
      else if (g.rank == 0)
        p.lane_slot[2 * li + (j & 1)] = lane_fetch(p, L.cls);
    }
    if (g.nb > 1) {
      if (!vg_sync(g, nullptr)) break;
      if (threadIdx.x == 0) s_idx = ld_acquire_i32(p.lane_slot + 2 * li + (j & 1));
    }
    __syncthreads();
    const int idx = s_idx;
    if (idx < 0) break;
    const BatchSys* __restrict__ S = p.sys + idx;
    if constexpr (PCG)
      pcg_mixed_body<float, false, ELL>(S->a, S->m, g);
    else
      bicgstab_mixed_body<float, false, ELL>(S->a, S->m, g);
    // a bounded wait of this system ran out: the lane stops (every block of
    // the lane sees the flag at its next barrier at the latest)
    if (ld_acquire_i32(&S->a.st->timeout) != 0) break;
  }
  if (p.lane_t && g.rank == 0 && threadIdx.x == 0) p.lane_t[2 * li + 1] = globaltimer_ns();
}

// f(std::integral_constant<int, OCC>{}) for the compiled occupancy nearest
// below occ (2 to 5 blocks per SM)
template <typename F>
const void* by_occ(int occ, F&& f) {
  switch (occ >= 5 ? 5 : occ) {
    case 5:
      return f(std::integral_constant<int, 5>{});
    case 4:
      return f(std::integral_constant<int, 4>{});
    case 3:
      return f(std::integral_constant<int, 3>{});
    default:
      return f(std::integral_constant<int, 2>{});
  }
}

// single-system solves also come in 6-8 blocks per SM (40 and 32 registers)
template <typename F>
const void* by_occ8(int occ, F&& f) {
  switch (occ >= 8 ? 8 : occ) {
    case 8:
      return f(std::integral_constant<int, 8>{});
    case 7:
      return f(std::integral_constant<int, 7>{});
    case 6:
      return f(std::integral_constant<int, 6>{});
    case 5:
      return f(std::integral_constant<int, 5>{});
    case 4:
      return f(std::integral_constant<int, 4>{});
    case 3:
      return f(std::integral_constant<int, 3>{});
    default:
      return f(std::integral_constant<int, 2>{});
  }
}

// ell: 0 CSR, 1 ELL, 2 ELL with the L2 prefetch of the next tile
const void* batch_kernel(bool pcg, int ell, int occ) {
  return by_occ(occ, [&](auto o) {
    constexpr int O = decltype(o)::value;
    if (pcg)
      return ell == 2 ? (const void*)k_mixed_batch<true, 2, O>
                      : ell == 1 ? (const void*)k_mixed_batch<true, 1, O> : (const void*)k_mixed_batch<true, 0, O>;
    return ell == 2 ? (const void*)k_mixed_batch<false, 2, O>
                    : ell == 1 ? (const void*)k_mixed_batch<false, 1, O> : (const void*)k_mixed_batch<false, 0, O>;
  });
}

}  // namespace

int launch_pcg_mixed(const KrylovArgs& a, const MixedArgs& m, cudaStream_t s) {
  const int ell = ell_mode(m);
  const void* one = ell == 0 ? (const void*)k_pcg_mixed<true, 0> : (const void*)k_pcg_mixed<true, 1>;
  const void* grid = by_occ8(g_mixed_occ, [&](auto o) {
    constexpr int O = decltype(o)::value;
    return ell == 2 ? (const void*)k_pcg_mixed<false, 2, O>
                    : ell == 1 ? (const void*)k_pcg_mixed<false, 1, O> : (const void*)k_pcg_mixed<false, 0, O>;
  });
  return launch_mixed(one, grid, a, m, s);
}

int launch_bicgstab_mixed(const KrylovArgs& a, const MixedArgs& m, cudaStream_t s) {
  const int ell = ell_mode(m);
  const void* one = ell == 0 ? (const void*)k_bicgstab_mixed<true, 0> : (const void*)k_bicgstab_mixed<true, 1>;
  const void* grid = by_occ8(g_mixed_occ, [&](auto o) {
    constexpr int O = decltype(o)::value;
    return ell == 2 ? (const void*)k_bicgstab_mixed<false, 2, O>
                    : ell == 1 ? (const void*)k_bicgstab_mixed<false, 1, O> : (const void*)k_bicgstab_mixed<false, 0, O>;
  });
  return launch_mixed(one, grid, a, m, s);
}

int batch_capacity(bool pcg, int ell) {
  constexpr int kDevs = 64;  // per device: the GPUs of a node may differ
  static int cap[kDevs][6][6] = {};
  const int idx = (pcg ? 3 : 0) + ell;
  const int occ = std::min(std::max(g_batch_occ, 2), 5);
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kDevs) dev = 0;
  if (cap[dev][idx][occ] == 0) {
    int sms = 0, per = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, batch_kernel(pcg, ell, occ), 256, 0);
    cap[dev][idx][occ] = sms * (per < 1 ? 1 : per);
  }
  return cap[dev][idx][occ];
}

int launch_mixed_batch(const LanePlan& p, bool pcg, int ell, cudaStream_t s) {
  if (p.nblocks <= 0) return 0;
  if (p.nblocks > batch_capacity(pcg, ell)) {
    set_error("batched solve: more blocks than can be co-resident");
    return MGPU_E_ARG;
  }
  cudaError_t e = cudaMemsetAsync(p.bars, 0, sizeof(unsigned long long) * (size_t)p.nlanes, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(p.q_head, 0, sizeof(int) * (size_t)p.ncls, s);
  if (e != cudaSuccess) return cuda_fail(e, "lane barrier reset", __FILE__, __LINE__);
  LanePlan pp = p;
  void* args[] = {(void*)&pp};
  e = cudaLaunchCooperativeKernel(batch_kernel(pcg, ell, g_batch_occ), dim3(p.nblocks), dim3(256), args, 0, s);
  if (e != cudaSuccess) return cuda_fail(e, "cooperative launch (batched)", __FILE__, __LINE__);
  return 0;
}

}  // namespace mgpu
