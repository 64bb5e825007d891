// noalloc.cu -- cg_jacobi on caller-owned device arrays, without allocating.
//
// Some callers cannot call cudaMalloc at all: a host that hands over only its
// own device buffers and forbids allocations behind its back (a memory pool or
// a framework that owns every byte of the device), or a CUDA Fortran host whose
// arrays already live on the GPU. For them this
// entry point runs the library's persistent PCG-Jacobi solve with every work
// vector, reduction partial, barrier counter and status word taken from one
// file-scope __device__ array of fixed size. The caller passes the matrix,
// the right-hand side and the solution as device pointers.
//
// Limits and rules:
//   * at most MGPU_NOALLOC_MAX_ROWS rows; larger systems are rejected;
//   * every GPU that loads the library holds the array (~4.9 MB) until exit;
//   * all calls share the one array, so calls that overlap on the GPU (two
//     streams, two host threads) race and corrupt each other; serialise them;
//   * the first call on a device looks the array's address up for that device
//     (cudaGetSymbolAddress);
//   * the call reads its result back and waits for its stream, so it cannot
//     run inside a stream capture;
//   * the solve's grid holds at most kPartials / 8 blocks (two halves of four
//     reduction partials per block); a larger grid is refused.

#include <cuda_runtime.h>

#include "case.cuh"

using namespace mgpu;

namespace {

constexpr long kMaxRows = MGPU_NOALLOC_MAX_ROWS;
constexpr long kPartials = 4 * 4096;
// layout in doubles: r z p q | diag (ints) | partials | barrier | status | record
constexpr long kOffDiag = 4 * kMaxRows;
constexpr long kOffPart = kOffDiag + kMaxRows / 2;
constexpr long kOffBar = kOffPart + kPartials;
constexpr long kOffStat = kOffBar + 4;
constexpr long kStatWords = (sizeof(DevStatus) + 7) / 8;
constexpr long kOffRec = kOffStat + kStatWords;
constexpr long kRecWords = (sizeof(MgpuIterRec) + 7) / 8;
constexpr long kOffFlags = kOffRec + kRecWords;
constexpr long kWords = kOffFlags + 4;

static __device__ __align__(256) double g_cg_scratch[kWords];

constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {nullptr};

// Diagonal positions of a 0-based CSR matrix; flags[0] = a row has no
// diagonal, flags[1] = b has a nonzero entry.
__global__ void k_find_diag(int n, const int* __restrict__ rp, const int* __restrict__ col,
                            const double* __restrict__ b, int* diag, int* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int d = -1;
  for (int k = rp[i]; k < rp[i + 1]; ++k)
    if (col[k] == i) {
      d = k;
      break;
    }
  diag[i] = d < 0 ? rp[i] : d;
  if (d < 0) atomicExch(&flags[0], 1);
  if (b[i] != 0.0) atomicExch(&flags[1], 1);
}

}  // namespace

extern "C" int mgpu_cg_jacobi_noalloc(int n, const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                      const double* d_val, const double* d_b, double* d_x, double tol, int maxit,
                                      int norm_mode, void* stream, int* it, double* res, int* ierr) {
  if (!d_row_ptr || !d_col_idx || !d_val || !d_b || !d_x || !it || !res || !ierr || maxit < 0 || n <= 0) {
    set_error("mgpu_cg_jacobi_noalloc: invalid argument");
    return MGPU_E_ARG;
  }
  if ((long)n > kMaxRows) {
    set_error("mgpu_cg_jacobi_noalloc: n = " + std::to_string(n) + " exceeds the fixed scratch limit of " +
              std::to_string(kMaxRows) + " rows; use mgpu_krylov_solve");
    return MGPU_E_ARG;
  }
  int dev = 0;
  MGPU_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("mgpu_cg_jacobi_noalloc: device id out of range");
    return MGPU_E_ARG;
  }
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    MGPU_CUDA(cudaGetSymbolAddress(&p, g_cg_scratch));
    g_scratch_addr[dev] = (double*)p;
  }
  double* S = g_scratch_addr[dev];
  cudaStream_t s = (cudaStream_t)stream;
  // state left by the previous call: status, record, flags start at zero
  MGPU_CUDA(cudaMemsetAsync(S + kOffStat, 0, sizeof(double) * (kWords - kOffStat), s));
  int* diag = (int*)(S + kOffDiag);
  int* flags = (int*)(S + kOffFlags);
  k_find_diag<<<ceil_div(n, 256), 256, 0, s>>>(n, d_row_ptr, d_col_idx, d_b, diag, flags);
  MGPU_LAUNCH_CHECK("k_find_diag");
  int hflags[2] = {0, 0};
  MGPU_CUDA(cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, s));
  MGPU_CUDA(cudaStreamSynchronize(s));
  *it = 0;
  *res = 0.0;
  *ierr = 0;
  if (hflags[0]) {  // cg_jacobi: b == 0 returns x = 0 first, else a missing diagonal is ierr 2
    if (!hflags[1]) {
      MGPU_CUDA(cudaMemsetAsync(d_x, 0, sizeof(double) * n, s));
      MGPU_CUDA(cudaStreamSynchronize(s));
    } else {
      *ierr = 2;
    }
    return 0;
  }
  KrylovArgs a{};
  a.n = n;
  a.row_ptr = d_row_ptr;
  a.col = d_col_idx;
  a.diag = diag;
  a.aval = d_val;
  a.b = d_b;
  a.x = d_x;
  a.r = S;
  a.z = S + kMaxRows;
  a.p = S + 2 * kMaxRows;
  a.v = S + 3 * kMaxRows;
  a.tol = tol;
  a.maxit = maxit;
  a.precond = 1;
  a.zero_x = 0;
  a.mpi_mode = norm_mode ? 1 : 0;
  a.partials = S + kOffPart;
  a.bar = (unsigned long long*)(S + kOffBar);
  a.st = (DevStatus*)(S + kOffStat);
  a.recs = (MgpuIterRec*)(S + kOffRec);
  a.slot = 0;
  a.ier_breakdown = 0;
  a.ferr = flags + 2;
  int block = 0;
  if (8l * krylov_grid(n, block, 0) > kPartials) {
    set_error("mgpu_cg_jacobi_noalloc: the solve's grid needs more reduction partials than the fixed array holds");
    return MGPU_E_ARG;
  }
  if (int e = launch_krylov_pcg(a, s)) return e;
  MgpuIterRec rec;
  DevStatus st;
  MGPU_CUDA(cudaMemcpyAsync(&rec, a.recs, sizeof(rec), cudaMemcpyDeviceToHost, s));
  MGPU_CUDA(cudaMemcpyAsync(&st, a.st, sizeof(st), cudaMemcpyDeviceToHost, s));
  MGPU_CUDA(cudaStreamSynchronize(s));
  if (st.timeout) {
    set_error("a bounded device wait ran out (grid barrier)");
    return MGPU_E_TIMEOUT;
  }
  *it = rec.lin_it[0];
  *res = rec.lin_res[0];
  *ierr = rec.lin_ierr[0];
  return 0;
}
