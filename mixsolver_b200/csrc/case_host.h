// case_host.h -- host-side state of a resident case and the driver helpers
// shared by the single-case runs (case.cu) and the batched runs (batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "assembly.cuh"
#include "case.cuh"

namespace mgpu {
// Non-blocking streams are recycled through a pool: creating and destroying
// one waits for kernels running on other streams, which stalls a case being
// set up or freed while a batch steps.
cudaStream_t acquire_stream();
void release_stream(cudaStream_t s);
// dst <- src through stream s, then a wait on s alone (a plain cudaMemcpy
// goes through the legacy default stream and waits for other streams' work).
int copy_sync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s);
}  // namespace mgpu

#define TRY(x)                 \
  do {                         \
    int rc_ = (x);             \
    if (rc_ != 0) return rc_;  \
  } while (0)

// A resident case: device arrays, parameters, its stream and run bookkeeping.
struct MgpuCase {
  using DeviceCase = mgpu::DeviceCase;
  using AsmParams = mgpu::AsmParams;
  DeviceCase d;
  AsmParams P;
  MgpuCtrl ctrl;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  int64_t bytes = 0;
  int has_outflow = 0;
  int profiling = 0;
  MgpuTiming timing{};
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  cudaEvent_t ev_run0 = nullptr, ev_run1 = nullptr;
  int64_t launches = 0;
  int kblock = 256;
  int run_mode = -1;  // batched runs: 0 SIMPLE, 1 PISO after mgpu_case_begin, -1 none
  int run_gen = 0;    // counts mgpu_case_begin calls
  double* stage = nullptr;  // device staging of cell-major field copies (grown on demand)
  size_t stage_n = 0;
  // mgpu_simple_run_fields: the last iteration's gp, gu and apc, final once
  // its gradients are formed, go to page-locked host arrays on copy_stream
  // while the iteration's pressure solve runs (gp and gu through stage2)
  struct EarlyCopy {
    double *gp = nullptr, *gu = nullptr, *apc = nullptr;
    bool armed = false, done = false;
  } early;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_early = nullptr, ev_copied = nullptr;
  double* stage2 = nullptr;
  size_t stage2_n = 0;
  std::vector<int> iface_faces;     // interface faces (0-based), bc order then face order
  int* d_iface_faces = nullptr;     // the same on the device

  template <typename T>
  int alloc(T*& p, size_t n) {
    p = nullptr;
    if (n == 0) n = 1;
    void* q = nullptr;
    // stream-ordered: freeing a case later never waits for other streams' work
    MGPU_CUDA(cudaMallocAsync(&q, n * sizeof(T), stream));
    allocs.push_back(q);
    bytes += (int64_t)(n * sizeof(T));
    p = (T*)q;
    return 0;
  }
  template <typename T>
  int upload(T*& p, const std::vector<T>& h) {
    if (int e = alloc(p, h.size())) return e;
    if (!h.empty()) MGPU_CUDA(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    return 0;
  }
  ~MgpuCase() {
    for (auto e : ev_pool) cudaEventDestroy(e);
    if (ev_run0) cudaEventDestroy(ev_run0);
    if (ev_run1) cudaEventDestroy(ev_run1);
    if (ev_copied) cudaEventSynchronize(ev_copied);
    if (ev_early) cudaEventDestroy(ev_early);
    if (ev_copied) cudaEventDestroy(ev_copied);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    for (void* p : allocs) cudaFreeAsync(p, stream);
    if (stage) cudaFreeAsync(stage, stream);
    if (stage2) cudaFreeAsync(stage2, stream);
    if (stream) mgpu::release_stream(stream);
  }
};

namespace mgpu {

extern int g_cheb_degree;
extern double g_cheb_ratio;
// the Chebyshev degree and interval ratio of a pressure solve of n rows
// (the cheb_* tuning keys; large systems take the large pair)
void cheb_params(long n, int& k, double& ratio);
extern int g_batch_reserve;
extern int g_prefetch_mb;
extern unsigned g_spin_limit;
extern unsigned g_poll_ns;

KrylovArgs base_args(MgpuCase* c);
MixedArgs mixed_args(const MgpuCase* c, bool bicg);
// momentum solve of component comp / pressure-correction solve into slot
KrylovArgs mom_args(MgpuCase* c, int comp, bool transient);
KrylovArgs ppe_args(MgpuCase* c, int slot, bool transient);
// one solve on stream s in the case's precision (FP64: factor + solve)
int krylov(MgpuCase* c, KrylovArgs a, bool bicg, cudaStream_t s);
// fresh device status for a run of nrec-1 iterations (ts_order 0 steady)
int reset_status(MgpuCase* c, int ts_order, int nrec);
int ensure_recs(MgpuCase* c, int n);
// device staging buffer of at least n doubles (stream-ordered, kept until the case is destroyed)
int ensure_stage(MgpuCase* c, size_t n);
// dst[planes*i + k] = src[q*n + i], q = k (grad: q = (k%3)*3 + k/3, the 3x3 gradient's transpose)
int launch_planes_to_cells(const double* src, long n, int planes, bool grad, double* dst, cudaStream_t s);
// dst[k*n + i] = src[planes*i + k]
int launch_cells_to_planes(const double* src, long n, int planes, double* dst, cudaStream_t s);

}  // namespace mgpu
