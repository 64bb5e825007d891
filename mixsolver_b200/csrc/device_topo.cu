// device_topo.cu -- the integer mesh pipeline and the reverse Cuthill-McKee
// cell order, built on the device.
//
// The arrays equal, entry for entry, what the host builder (mesh_host.cpp)
// and the reference give:
//   * cell -> face lists in ascending face order and the cell -> cell lists
//     in face order (build_connectivity, mod_uns_connectivity.f90:28-108):
//     one radix sort of (cell, face) keys each;
//   * the CSR pattern of build_cell_csr (mod_uns_simple.f90:835-887): the
//     (cell, neighbour) pairs plus the diagonal, sorted and made unique;
//   * the diagonal positions, the face -> CSR-slot map (pos_of,
//     mod_uns_simple.f90:909-923) and the transpose map, by binary search in
//     the sorted rows;
//   * the level sets of the strictly lower and upper triangles: level(i) =
//     1 + the largest level of the rows row i depends on, relaxed to its fixed
//     point in parallel sweeps (it only grows, and the longest path is the
//     unique fixed point), then rows bucketed by (level, row);
//   * the reverse Cuthill-McKee order of mgpu_rcm_order: George-Liu start
//     (level-synchronous BFS, the last level's least (degree, index) cell),
//     then Cuthill-McKee level by level. Within a level the serial algorithm
//     appends each cell when its first-visited neighbour of the previous level
//     is processed, children of one parent in (degree, index) order; so a
//     level is the sort of its cells by (position of that parent, degree,
//     index), the parent being the least-positioned neighbour (atomicMin).
// Sorts, scans and compactions come from CUB (cub::DeviceRadixSort,
// cub::DeviceScan, cub::DeviceSelect); the kernels are this file's.

#include <cuda_runtime.h>

#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <vector>

#include "device_topo.h"
#include "mesh_host.h"

namespace mgpu {
namespace {

using u64 = unsigned long long;

// Stream-ordered temporaries of one call, freed at scope exit.
struct Tmp {
  cudaStream_t s;
  std::vector<void*> p;
  explicit Tmp(cudaStream_t st) : s(st) {}
  ~Tmp() {
    for (void* q : p) cudaFreeAsync(q, s);
  }
  template <typename T>
  int get(T*& out, size_t n) {
    void* q = nullptr;
    MGPU_CUDA(cudaMallocAsync(&q, sizeof(T) * std::max<size_t>(n, 1), s));
    p.push_back(q);
    out = (T*)q;
    return 0;
  }
};

#define DT_TRY(x)             \
  do {                        \
    int rc_ = (x);            \
    if (rc_ != 0) return rc_; \
  } while (0)

int bits_for(long v) {
  int b = 1;
  while ((1l << b) <= v) ++b;
  return b;
}

int sort_keys(Tmp& T, const u64* in, u64* out, int n, int end_bit) {
  if (n <= 0) return 0;
  size_t bytes = 0;
  MGPU_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, bytes, in, out, n, 0, end_bit, T.s));
  char* tmp = nullptr;
  DT_TRY(T.get(tmp, bytes));
  MGPU_CUDA(cub::DeviceRadixSort::SortKeys(tmp, bytes, in, out, n, 0, end_bit, T.s));
  return 0;
}

int sort_pairs(Tmp& T, const u64* kin, u64* kout, const int* vin, int* vout, int n, int end_bit) {
  if (n <= 0) return 0;
  size_t bytes = 0;
  MGPU_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, 0, end_bit, T.s));
  char* tmp = nullptr;
  DT_TRY(T.get(tmp, bytes));
  MGPU_CUDA(cub::DeviceRadixSort::SortPairs(tmp, bytes, kin, kout, vin, vout, n, 0, end_bit, T.s));
  return 0;
}

// ptr[0..n] = exclusive sum of cnt[0..n) (cnt has n + 1 entries, the last 0)
int scan_counts(Tmp& T, const int* cnt, int* ptr, int n) {
  size_t bytes = 0;
  MGPU_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt, ptr, n + 1, T.s));
  char* tmp = nullptr;
  DT_TRY(T.get(tmp, bytes));
  MGPU_CUDA(cub::DeviceScan::ExclusiveSum(tmp, bytes, cnt, ptr, n + 1, T.s));
  return 0;
}

int read_int(const int* d, int& h, cudaStream_t s) {
  MGPU_CUDA(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, s));
  MGPU_CUDA(cudaStreamSynchronize(s));
  return 0;
}

// ---------------- connectivity -------------------------------------------

// (cell, face) keys of every face side: owner side at i, neighbour side at
// F + i (a boundary face's second key sorts past every cell and is dropped);
// cnt[cell] counts the sides of each cell
__global__ void k_face_keys(int F, int N, const int* __restrict__ c0, const int* __restrict__ c1, u64* keys,
                            int* cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F) return;
  const int a = c0[i], b = c1[i];
  keys[i] = ((u64)a << 32) | (u64)i;
  atomicAdd(&cnt[a], 1);
  if (b >= 0) {
    keys[F + i] = ((u64)b << 32) | (u64)i;
    atomicAdd(&cnt[b], 1);
  } else {
    keys[F + i] = ((u64)N << 32) | (u64)i;
  }
}

// (cell, face) keys of interior face sides with the cell across as value
__global__ void k_nbr_keys(int F, int N, const int* __restrict__ c0, const int* __restrict__ c1, u64* keys,
                           int* vals, int* cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= F) return;
  const int a = c0[i], b = c1[i];
  if (b >= 0) {
    keys[i] = ((u64)a << 32) | (u64)i;
    vals[i] = b;
    keys[F + i] = ((u64)b << 32) | (u64)i;
    vals[F + i] = a;
    atomicAdd(&cnt[a], 1);
    atomicAdd(&cnt[b], 1);
  } else {
    keys[i] = ((u64)N << 32) | (u64)i;
    keys[F + i] = ((u64)N << 32) | (u64)i;
    vals[i] = vals[F + i] = -1;
  }
}

__global__ void k_low_word(long n, const u64* __restrict__ keys, int* out) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k < n) out[k] = (int)(keys[k] & 0xffffffffull);
}

// (cell, column) keys of the CSR pattern: the neighbour entries, then the diagonals
__global__ void k_pattern_keys(int N, int ncc, const int* __restrict__ c2c_ptr, const int* __restrict__ c2c,
                               u64* keys) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  for (int k = c2c_ptr[c]; k < c2c_ptr[c + 1]; ++k) keys[k] = ((u64)c << 32) | (u64)(unsigned)c2c[k];
  keys[ncc + c] = ((u64)c << 32) | (u64)c;
}

__global__ void k_pattern_rows(int nnz, const u64* __restrict__ keys, int* cnt, int* col) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nnz) return;
  col[k] = (int)(keys[k] & 0xffffffffull);
  atomicAdd(&cnt[(int)(keys[k] >> 32)], 1);
}

__device__ __forceinline__ int find_in_row(const int* __restrict__ rp, const int* __restrict__ col, int i, int j) {
  int lo = rp[i], hi = rp[i + 1];
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (col[mid] < j)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < rp[i + 1] && col[lo] == j) ? lo : -1;
}

__global__ void k_diag_slots(int N, const int* __restrict__ rp, const int* __restrict__ col, const int* __restrict__ cf_ptr,
                             const int* __restrict__ cf, const int* __restrict__ c0, const int* __restrict__ c1,
                             int* diag, int* cf_slot) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  diag[c] = find_in_row(rp, col, c, c);
  for (int k = cf_ptr[c]; k < cf_ptr[c + 1]; ++k) {
    const int f = cf[k];
    if (c1[f] < 0) {
      cf_slot[k] = -1;
      continue;
    }
    const int other = (c0[f] == c) ? c1[f] : c0[f];
    cf_slot[k] = find_in_row(rp, col, c, other);
  }
}

__global__ void k_mirror(int N, const int* __restrict__ rp, const int* __restrict__ col, int* mirror) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  for (int k = rp[i]; k < rp[i + 1]; ++k) mirror[k] = find_in_row(rp, col, col[k], i);
}

// ---------------- level sets ----------------------------------------------

// one relaxation sweep: LOWER uses the entries left of the diagonal, else right
template <bool LOWER>
__global__ void k_level_sweep(int N, const int* __restrict__ rp, const int* __restrict__ col,
                              const int* __restrict__ diag, int* lev, int* changed) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int b = LOWER ? rp[i] : diag[i] + 1, e = LOWER ? diag[i] : rp[i + 1];
  int l = 0;
  for (int k = b; k < e; ++k) l = max(l, ((volatile int*)lev)[col[k]] + 1);
  if (l != lev[i]) {
    lev[i] = l;
    *changed = 1;
  }
}

__global__ void k_level_keys(int N, const int* __restrict__ lev, u64* keys, int* cnt, int* nlev) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  keys[i] = ((u64)lev[i] << 32) | (u64)i;
  atomicAdd(&cnt[lev[i]], 1);
  atomicMax(nlev, lev[i] + 1);
}

int level_sets(Tmp& T, int N, const int* rp, const int* col, const int* diag, bool lower, DeviceTopo& t,
               const TopoAlloc& alloc) {
  cudaStream_t s = T.s;
  int *lev = nullptr, *flag = nullptr;
  DT_TRY(T.get(lev, N));
  DT_TRY(T.get(flag, 2));
  MGPU_CUDA(cudaMemsetAsync(lev, 0, sizeof(int) * (size_t)N, s));
  const unsigned g = ceil_div(N, 256);
  for (int round = 0;; ++round) {
    MGPU_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
    for (int k = 0; k < 8; ++k) {  // a few sweeps per look at the flag
      if (lower)
        k_level_sweep<true><<<g, 256, 0, s>>>(N, rp, col, diag, lev, flag);
      else
        k_level_sweep<false><<<g, 256, 0, s>>>(N, rp, col, diag, lev, flag);
    }
    MGPU_LAUNCH_CHECK("k_level_sweep");
    int changed = 0;
    DT_TRY(read_int(flag, changed, s));
    if (!changed) break;
    if (round > N) {
      set_error("device topology: level sets did not settle");
      return MGPU_E_MESH;
    }
  }
  int *cnt = nullptr;
  DT_TRY(T.get(cnt, N + 1));
  MGPU_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(N + 1), s));
  MGPU_CUDA(cudaMemsetAsync(flag + 1, 0, sizeof(int), s));
  u64 *keys = nullptr, *sorted = nullptr;
  DT_TRY(T.get(keys, N));
  DT_TRY(T.get(sorted, N));
  k_level_keys<<<g, 256, 0, s>>>(N, lev, keys, cnt, flag + 1);
  MGPU_LAUNCH_CHECK("k_level_keys");
  int nlev = 0;
  DT_TRY(read_int(flag + 1, nlev, s));
  DT_TRY(sort_keys(T, keys, sorted, N, 32 + bits_for(nlev)));
  int *ptr = nullptr, *rows = nullptr;
  DT_TRY(alloc(ptr, nlev + 1));
  DT_TRY(alloc(rows, N));
  DT_TRY(scan_counts(T, cnt, ptr, nlev));
  k_low_word<<<g, 256, 0, s>>>(N, sorted, rows);
  MGPU_LAUNCH_CHECK("k_low_word");
  if (lower) {
    t.nlev_lo = nlev;
    t.lo_ptr = ptr;
    t.lo_rows = rows;
  } else {
    t.nlev_up = nlev;
    t.up_ptr = ptr;
    t.up_rows = rows;
  }
  return 0;
}

// ---------------- reverse Cuthill-McKee -----------------------------------

__global__ void k_degree(int N, const int* __restrict__ rp, int* deg, int* maxdeg) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  deg[c] = rp[c + 1] - rp[c] - 1;
  atomicMax(maxdeg, deg[c]);
}

// least (degree, index) over the unvisited cells
__global__ void k_least_unvisited(int N, const int* __restrict__ deg, const int* __restrict__ visited, u64* best) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N || visited[c]) return;
  atomicMin(best, ((u64)deg[c] << 32) | (u64)c);
}

// least (degree, index) over a list of cells
__global__ void k_least_of(int n, const int* __restrict__ list, const int* __restrict__ deg, u64* best) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int c = list[t];
  atomicMin(best, ((u64)deg[c] << 32) | (u64)c);
}

// one BFS level among the unvisited cells (order within a level irrelevant)
__global__ void k_bfs_level(int n, const int* __restrict__ cur, const int* __restrict__ rp, const int* __restrict__ col,
                            const int* __restrict__ visited, int* mark, int stamp, int* next, int* cnt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int v = cur[t];
  for (int k = rp[v]; k < rp[v + 1]; ++k) {
    const int w = col[k];
    if (w == v || visited[w]) continue;
    if (atomicExch(&mark[w], stamp) != stamp) next[atomicAdd(cnt, 1)] = w;
  }
}

// Cuthill-McKee: the cells of the next level with the least position of a
// current-level neighbour (the parent that appends them)
__global__ void k_cm_expand(int n, int off, const int* __restrict__ cur, const int* __restrict__ rp,
                            const int* __restrict__ col, const int* __restrict__ visited, int* parent, int* mark,
                            int stamp, int* next, int* cnt) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int v = cur[t];
  for (int k = rp[v]; k < rp[v + 1]; ++k) {
    const int w = col[k];
    if (w == v || visited[w]) continue;
    atomicMin(&parent[w], off + t);
    if (atomicExch(&mark[w], stamp) != stamp) next[atomicAdd(cnt, 1)] = w;
  }
}

// sort key of a next-level cell: (parent position, degree, index); positions
// and indices below 2^24, degrees below 2^8
__global__ void k_cm_keys(int n, const int* __restrict__ next, const int* __restrict__ parent,
                          const int* __restrict__ deg, u64* keys) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int w = next[t];
  keys[t] = ((u64)parent[w] << 32) | ((u64)deg[w] << 24) | (u64)w;
}

__global__ void k_cm_place(int n, int off, const u64* __restrict__ keys, int* order, int* visited, int* cur) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int w = (int)(keys[t] & 0xffffffull);
  order[off + t] = w;
  cur[t] = w;
  visited[w] = 1;
}

__global__ void k_reverse(int N, const int* __restrict__ order, int* new_of_old) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  new_of_old[order[N - 1 - p]] = p + 1;
}

// ---------------- per-case lists ------------------------------------------

__global__ void k_row_width(int N, const int* __restrict__ rp, int* w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) atomicMax(w, rp[i + 1] - rp[i]);
}

// column-major ELL pattern: entry t of row i at t * ld + i, padding the row
// itself (rows ld > i >= N: the last row)
__global__ void k_ell_pattern(int N, int W, long ld, const int* __restrict__ rp, const int* __restrict__ col,
                              int* ell) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= ld) return;
  if (i >= N) {
    for (int t = 0; t < W; ++t) ell[t * ld + i] = N - 1;
    return;
  }
  const int b = rp[i], e = rp[i + 1];
  for (int t = 0; t < W; ++t) ell[t * ld + i] = b + t < e ? col[b + t] : (int)i;
}

__global__ void k_bface_count(int N, const int* __restrict__ cf_ptr, const int* __restrict__ cf,
                              const int* __restrict__ c1, const int* __restrict__ fgrp, int* cnt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  int n = 0;
  for (int k = cf_ptr[c]; k < cf_ptr[c + 1]; ++k) {
    const int f = cf[k];
    if (c1[f] < 0 && fgrp[f] >= 0) ++n;
  }
  cnt[c] = n;
}

__global__ void k_bface_fill(int N, const int* __restrict__ cf_ptr, const int* __restrict__ cf,
                             const int* __restrict__ c1, const int* __restrict__ fgrp, const int* __restrict__ bptr,
                             int* bf) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  int j = bptr[c];
  for (int k = cf_ptr[c]; k < cf_ptr[c + 1]; ++k) {
    const int f = cf[k];
    if (c1[f] < 0 && fgrp[f] >= 0) bf[j++] = f;
  }
}

}  // namespace

int device_topology(int N, int F, const int* c0, const int* c1, DeviceTopo& t, const TopoAlloc& alloc,
                    cudaStream_t s, bool levels) {
  Tmp T(s);
  t.N = N;
  t.F = F;
  const unsigned gF = ceil_div(F, 256), gN = ceil_div(N, 256);
  const int cbits = 32 + bits_for(N);  // keys (cell, face) with cell <= N
  // cell -> faces
  u64 *keys = nullptr, *sorted = nullptr;
  int *cnt = nullptr;
  DT_TRY(T.get(keys, 2l * F));
  DT_TRY(T.get(sorted, 2l * F));
  DT_TRY(T.get(cnt, N + 1));
  MGPU_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(N + 1), s));
  k_face_keys<<<gF, 256, 0, s>>>(F, N, c0, c1, keys, cnt);
  MGPU_LAUNCH_CHECK("k_face_keys");
  DT_TRY(sort_keys(T, keys, sorted, 2 * F, cbits));
  DT_TRY(alloc(t.cf_ptr, N + 1));
  DT_TRY(scan_counts(T, cnt, t.cf_ptr, N));
  int ncf = 0;
  DT_TRY(read_int(t.cf_ptr + N, ncf, s));
  DT_TRY(alloc(t.cf, ncf));
  k_low_word<<<ceil_div(ncf, 256), 256, 0, s>>>(ncf, sorted, t.cf);
  MGPU_LAUNCH_CHECK("k_low_word");
  t.ncf = ncf;
  // cell -> cells (face order)
  int *vals = nullptr, *svals = nullptr;
  DT_TRY(T.get(vals, 2l * F));
  DT_TRY(T.get(svals, 2l * F));
  MGPU_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(N + 1), s));
  k_nbr_keys<<<gF, 256, 0, s>>>(F, N, c0, c1, keys, vals, cnt);
  MGPU_LAUNCH_CHECK("k_nbr_keys");
  DT_TRY(sort_pairs(T, keys, sorted, vals, svals, 2 * F, cbits));
  DT_TRY(alloc(t.c2c_ptr, N + 1));
  DT_TRY(scan_counts(T, cnt, t.c2c_ptr, N));
  int ncc = 0;
  DT_TRY(read_int(t.c2c_ptr + N, ncc, s));
  DT_TRY(alloc(t.c2c, ncc));
  if (ncc > 0) MGPU_CUDA(cudaMemcpyAsync(t.c2c, svals, sizeof(int) * (size_t)ncc, cudaMemcpyDeviceToDevice, s));
  t.ncc = ncc;
  // CSR pattern: self + unique neighbours, ascending
  u64 *pkeys = nullptr, *psorted = nullptr, *puniq = nullptr;
  int* nsel = nullptr;
  DT_TRY(T.get(pkeys, (size_t)ncc + N));
  DT_TRY(T.get(psorted, (size_t)ncc + N));
  DT_TRY(T.get(puniq, (size_t)ncc + N));
  DT_TRY(T.get(nsel, 1));
  k_pattern_keys<<<gN, 256, 0, s>>>(N, ncc, t.c2c_ptr, t.c2c, pkeys);
  MGPU_LAUNCH_CHECK("k_pattern_keys");
  DT_TRY(sort_keys(T, pkeys, psorted, ncc + N, 32 + bits_for(N)));
  {
    size_t bytes = 0;
    MGPU_CUDA(cub::DeviceSelect::Unique(nullptr, bytes, psorted, puniq, nsel, ncc + N, s));
    char* tmp = nullptr;
    DT_TRY(T.get(tmp, bytes));
    MGPU_CUDA(cub::DeviceSelect::Unique(tmp, bytes, psorted, puniq, nsel, ncc + N, s));
  }
  int nnz = 0;
  DT_TRY(read_int(nsel, nnz, s));
  t.nnz = nnz;
  DT_TRY(alloc(t.col, nnz));
  DT_TRY(alloc(t.row_ptr, N + 1));
  MGPU_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(N + 1), s));
  k_pattern_rows<<<ceil_div(nnz, 256), 256, 0, s>>>(nnz, puniq, cnt, t.col);
  MGPU_LAUNCH_CHECK("k_pattern_rows");
  DT_TRY(scan_counts(T, cnt, t.row_ptr, N));
  // diagonal, face -> slot, transpose
  DT_TRY(alloc(t.diag, N));
  DT_TRY(alloc(t.cf_slot, ncf));
  DT_TRY(alloc(t.mirror, nnz));
  k_diag_slots<<<gN, 256, 0, s>>>(N, t.row_ptr, t.col, t.cf_ptr, t.cf, c0, c1, t.diag, t.cf_slot);
  MGPU_LAUNCH_CHECK("k_diag_slots");
  k_mirror<<<gN, 256, 0, s>>>(N, t.row_ptr, t.col, t.mirror);
  MGPU_LAUNCH_CHECK("k_mirror");
  // level sets of the triangular sweeps
  if (levels) {
    DT_TRY(level_sets(T, N, t.row_ptr, t.col, t.diag, true, t, alloc));
    DT_TRY(level_sets(T, N, t.row_ptr, t.col, t.diag, false, t, alloc));
  }
  MGPU_CUDA(cudaStreamSynchronize(s));
  return 0;
}

int device_ell(int N, const int* rp, const int* col, int max_width, int& W, long& ld, int*& ell,
               const TopoAlloc& alloc, cudaStream_t s) {
  Tmp T(s);
  int* w = nullptr;
  DT_TRY(T.get(w, 1));
  MGPU_CUDA(cudaMemsetAsync(w, 0, sizeof(int), s));
  k_row_width<<<ceil_div(N, 256), 256, 0, s>>>(N, rp, w);
  MGPU_LAUNCH_CHECK("k_row_width");
  DT_TRY(read_int(w, W, s));
  ell = nullptr;
  ld = ((long)N + 3) / 4 * 4;  // each column starts on a 16-byte boundary
  if (W > max_width) return 0;
  DT_TRY(alloc(ell, (size_t)W * ld));
  k_ell_pattern<<<ceil_div(ld, 256), 256, 0, s>>>(N, W, ld, rp, col, ell);
  MGPU_LAUNCH_CHECK("k_ell_pattern");
  return 0;
}

int device_boundary_lists(int N, const int* cf_ptr, const int* cf, const int* c1, const int* fgrp, int*& bf_ptr,
                          int*& bf, const TopoAlloc& alloc, cudaStream_t s) {
  Tmp T(s);
  int* cnt = nullptr;
  DT_TRY(T.get(cnt, N + 1));
  MGPU_CUDA(cudaMemsetAsync(cnt + N, 0, sizeof(int), s));
  const unsigned g = ceil_div(N, 256);
  k_bface_count<<<g, 256, 0, s>>>(N, cf_ptr, cf, c1, fgrp, cnt);
  MGPU_LAUNCH_CHECK("k_bface_count");
  DT_TRY(alloc(bf_ptr, N + 1));
  DT_TRY(scan_counts(T, cnt, bf_ptr, N));
  int nb = 0;
  DT_TRY(read_int(bf_ptr + N, nb, s));
  DT_TRY(alloc(bf, nb));
  k_bface_fill<<<g, 256, 0, s>>>(N, cf_ptr, cf, c1, fgrp, bf_ptr, bf);
  MGPU_LAUNCH_CHECK("k_bface_fill");
  return 0;
}

int device_rcm(int N, const int* rp, const int* col, int* new_of_old, cudaStream_t s) {
  if (N <= 0 || N >= (1 << 24)) {
    set_error("device RCM: at most 2^24 - 1 cells");
    return MGPU_E_ARG;
  }
  Tmp T(s);
  const unsigned gN = ceil_div(N, 256);
  int *deg = nullptr, *visited = nullptr, *mark = nullptr, *parent = nullptr, *order = nullptr;
  int *cur = nullptr, *next = nullptr, *cnt = nullptr;
  u64 *best = nullptr, *keys = nullptr, *skeys = nullptr;
  DT_TRY(T.get(deg, N));
  DT_TRY(T.get(visited, N));
  DT_TRY(T.get(mark, N));
  DT_TRY(T.get(parent, N));
  DT_TRY(T.get(order, N));
  DT_TRY(T.get(cur, N));
  DT_TRY(T.get(next, N));
  DT_TRY(T.get(cnt, 2));
  DT_TRY(T.get(best, 1));
  DT_TRY(T.get(keys, N));
  DT_TRY(T.get(skeys, N));
  MGPU_CUDA(cudaMemsetAsync(visited, 0, sizeof(int) * (size_t)N, s));
  MGPU_CUDA(cudaMemsetAsync(mark, 0, sizeof(int) * (size_t)N, s));
  MGPU_CUDA(cudaMemsetAsync(parent, 0x7f, sizeof(int) * (size_t)N, s));
  MGPU_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * 2, s));
  k_degree<<<gN, 256, 0, s>>>(N, rp, deg, cnt + 1);
  MGPU_LAUNCH_CHECK("k_degree");
  int maxdeg = 0;
  DT_TRY(read_int(cnt + 1, maxdeg, s));
  if (maxdeg >= 256) {
    set_error("device RCM: a cell with 256 or more neighbours");
    return MGPU_E_ARG;
  }
  auto least = [&](bool list, int n, const int* l, int& cell) -> int {
    const u64 init = ~0ull;
    MGPU_CUDA(cudaMemcpyAsync(best, &init, sizeof(u64), cudaMemcpyHostToDevice, s));
    if (list)
      k_least_of<<<ceil_div(n, 256), 256, 0, s>>>(n, l, deg, best);
    else
      k_least_unvisited<<<gN, 256, 0, s>>>(N, deg, visited, best);
    MGPU_LAUNCH_CHECK("k_least");
    u64 h = 0;
    MGPU_CUDA(cudaMemcpyAsync(&h, best, sizeof(u64), cudaMemcpyDeviceToHost, s));
    MGPU_CUDA(cudaStreamSynchronize(s));
    cell = (int)(h & 0xffffffffull);
    return 0;
  };
  int stamp = 0;
  // BFS from r among the unvisited cells: eccentricity and the least
  // (degree, index) cell of the last level
  auto bfs = [&](int r, int& ecc, int& xlast) -> int {
    ++stamp;
    MGPU_CUDA(cudaMemcpyAsync(cur, &r, sizeof(int), cudaMemcpyHostToDevice, s));
    MGPU_CUDA(cudaMemcpyAsync(mark + r, &stamp, sizeof(int), cudaMemcpyHostToDevice, s));
    int n = 1;
    ecc = 0;
    int* a = cur;
    int* b = next;
    while (true) {
      MGPU_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), s));
      k_bfs_level<<<ceil_div(n, 256), 256, 0, s>>>(n, a, rp, col, visited, mark, stamp, b, cnt);
      MGPU_LAUNCH_CHECK("k_bfs_level");
      int m = 0;
      DT_TRY(read_int(cnt, m, s));
      if (m == 0) break;
      ++ecc;
      std::swap(a, b);
      n = m;
    }
    return least(true, n, a, xlast);
  };
  int placed = 0;
  while (placed < N) {
    int r = 0, ecc = 0, x = 0;
    DT_TRY(least(false, 0, nullptr, r));
    DT_TRY(bfs(r, ecc, x));
    while (true) {
      int ex = 0, xx = 0;
      DT_TRY(bfs(x, ex, xx));
      if (ex > ecc) {
        r = x;
        ecc = ex;
        x = xx;
      } else {
        break;
      }
    }
    // Cuthill-McKee from r, level by level
    const int one = 1;
    MGPU_CUDA(cudaMemcpyAsync(order + placed, &r, sizeof(int), cudaMemcpyHostToDevice, s));
    MGPU_CUDA(cudaMemcpyAsync(cur, &r, sizeof(int), cudaMemcpyHostToDevice, s));
    MGPU_CUDA(cudaMemcpyAsync(visited + r, &one, sizeof(int), cudaMemcpyHostToDevice, s));
    int off = placed, n = 1;
    placed += 1;
    while (true) {
      ++stamp;
      MGPU_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int), s));
      k_cm_expand<<<ceil_div(n, 256), 256, 0, s>>>(n, off, cur, rp, col, visited, parent, mark, stamp, next, cnt);
      MGPU_LAUNCH_CHECK("k_cm_expand");
      int m = 0;
      DT_TRY(read_int(cnt, m, s));
      if (m == 0) break;
      k_cm_keys<<<ceil_div(m, 256), 256, 0, s>>>(m, next, parent, deg, keys);
      MGPU_LAUNCH_CHECK("k_cm_keys");
      DT_TRY(sort_keys(T, keys, skeys, m, 32 + bits_for(placed)));
      k_cm_place<<<ceil_div(m, 256), 256, 0, s>>>(m, placed, skeys, order, visited, cur);
      MGPU_LAUNCH_CHECK("k_cm_place");
      off = placed;
      placed += m;
      n = m;
    }
  }
  k_reverse<<<gN, 256, 0, s>>>(N, order, new_of_old);
  MGPU_LAUNCH_CHECK("k_reverse");
  MGPU_CUDA(cudaStreamSynchronize(s));
  return 0;
}

}  // namespace mgpu

// ---------------- C-ABI -----------------------------------------------------

namespace {

using namespace mgpu;

// one stream and the device arrays of one mesh-pipeline call
struct MeshCall {
  cudaStream_t s = nullptr;
  std::vector<void*> keep;
  ~MeshCall() {
    for (void* p : keep) cudaFreeAsync(p, s);
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
  int init() {
    MGPU_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    return 0;
  }
  TopoAlloc allocator() {
    return [this](int*& p, size_t n) -> int {
      void* q = nullptr;
      MGPU_CUDA(cudaMallocAsync(&q, sizeof(int) * std::max<size_t>(n, 1), s));
      keep.push_back(q);
      p = (int*)q;
      return 0;
    };
  }
  int up(int*& d, const std::vector<int>& h) {
    DT_TRY(allocator()(d, h.size()));
    if (!h.empty()) MGPU_CUDA(cudaMemcpyAsync(d, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice, s));
    return 0;
  }
  int down(int32_t* h, const int* d, long n) {
    if (h && n > 0) MGPU_CUDA(cudaMemcpyAsync(h, d, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, s));
    return 0;
  }
};

}  // namespace

extern "C" {

int mgpu_mesh_topology(const MgpuMesh* mesh, int on_device, int32_t* sizes, int32_t* cf_ptr, int32_t* cf,
                       int32_t* row_ptr, int32_t* col, int32_t* diag, int32_t* cf_slot, int32_t* lt_pos,
                       int32_t* lo_ptr, int32_t* lo_rows, int32_t* up_ptr, int32_t* up_rows) {
  if (!sizes) return MGPU_E_ARG;
  HostMesh m;
  std::string why;
  if (int e = load_host_mesh(mesh, m, why)) {
    set_error(why);
    return e;
  }
  const int N = m.N;
  if (!on_device) {
    HostTopo t;
    build_topology(m, t);
    sizes[0] = (int)t.cf.size();
    sizes[1] = (int)t.col.size();
    sizes[2] = t.nlev_lo;
    sizes[3] = t.nlev_up;
    auto put = [](int32_t* h, const std::vector<int>& v) {
      if (h) std::copy(v.begin(), v.end(), h);
    };
    put(cf_ptr, t.cf_ptr);
    put(cf, t.cf);
    put(row_ptr, t.row_ptr);
    put(col, t.col);
    put(diag, t.diag);
    put(cf_slot, t.cf_slot);
    put(lt_pos, t.mirror);
    put(lo_ptr, t.lo_ptr);
    put(lo_rows, t.lo_rows);
    put(up_ptr, t.up_ptr);
    put(up_rows, t.up_rows);
    return 0;
  }
  MeshCall C;
  DT_TRY(C.init());
  int *dc0 = nullptr, *dc1 = nullptr;
  DT_TRY(C.up(dc0, m.c0));
  DT_TRY(C.up(dc1, m.c1));
  DeviceTopo t;
  DT_TRY(device_topology(N, m.F, dc0, dc1, t, C.allocator(), C.s));
  sizes[0] = t.ncf;
  sizes[1] = t.nnz;
  sizes[2] = t.nlev_lo;
  sizes[3] = t.nlev_up;
  DT_TRY(C.down(cf_ptr, t.cf_ptr, N + 1));
  DT_TRY(C.down(cf, t.cf, t.ncf));
  DT_TRY(C.down(row_ptr, t.row_ptr, N + 1));
  DT_TRY(C.down(col, t.col, t.nnz));
  DT_TRY(C.down(diag, t.diag, N));
  DT_TRY(C.down(cf_slot, t.cf_slot, t.ncf));
  DT_TRY(C.down(lt_pos, t.mirror, t.nnz));
  DT_TRY(C.down(lo_ptr, t.lo_ptr, t.nlev_lo + 1));
  DT_TRY(C.down(lo_rows, t.lo_rows, N));
  DT_TRY(C.down(up_ptr, t.up_ptr, t.nlev_up + 1));
  DT_TRY(C.down(up_rows, t.up_rows, N));
  MGPU_CUDA(cudaStreamSynchronize(C.s));
  return 0;
}

int mgpu_rcm_order_device(const MgpuMesh* mesh, int32_t* new_of_old) {
  if (!new_of_old) return MGPU_E_ARG;
  HostMesh m;
  std::string why;
  if (int e = load_host_mesh(mesh, m, why)) {
    set_error(why);
    return e;
  }
  MeshCall C;
  DT_TRY(C.init());
  int *dc0 = nullptr, *dc1 = nullptr, *dout = nullptr;
  DT_TRY(C.up(dc0, m.c0));
  DT_TRY(C.up(dc1, m.c1));
  DeviceTopo t;
  DT_TRY(device_topology(m.N, m.F, dc0, dc1, t, C.allocator(), C.s));
  DT_TRY(C.allocator()(dout, m.N));
  DT_TRY(device_rcm(m.N, t.row_ptr, t.col, dout, C.s));
  DT_TRY(C.down(new_of_old, dout, m.N));
  MGPU_CUDA(cudaStreamSynchronize(C.s));
  return 0;
}

}  // extern "C"
