// batch.cu -- many resident cases advanced together.
//
// The reference runs one case per process (simple_run / piso_run_mpi). Here a
// batch advances any number of resident cases of uneven size in lock step,
// one outer iteration (SIMPLE) or time step (PISO) at a time:
//   * every assembly kernel is ONE launch over all cases (kb_* in
//     assembly.cu): block b works for the case blk_case[b] and computes
//     exactly what that case's own launch computes;
//   * every Krylov phase (momentum component 0, 1, 2; pressure corrector
//     0..n-1) is ONE persistent cooperative launch over all mixed-precision
//     systems, split into lanes (k_mixed_batch in krylov_mixed.cu); FP64
//     cases are solved one after the other by the single-case kernels;
//   * the whole iteration is captured once in a CUDA graph and replayed.
// Cases that have converged, failed or reached their iteration count drop out
// on the device (their kernels return at once), so a step never waits on the
// host.
//
// Lane plan (the tiling and chunking): the mixed-precision solves give the
// same result on any number of blocks, so the plan is free to balance. Systems
// above a row threshold run on a few wide lanes that share their class's
// blocks; the others on single-block lanes; the blocks are split by each
// class's share of the work (modelled on the first iteration, measured
// iteration counts after it). Which lane solves which system is decided at run
// time: each class has a queue of its systems, most work first, a lane takes
// the next one of its class, and wide lanes take small systems once theirs are
// done. With autotuning on, the first pressure solve of a batch is timed under
// each candidate (threshold, wide lanes) and the fastest is kept.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <string>
#include <vector>

#include "assembly.cuh"
#include "case.cuh"
#include "case_host.h"

using namespace mgpu;

namespace {

// Lane policy: systems of more than split_rows rows run on wide lanes (one
// lane per big system, sized by its work, when there are at most wide_lanes of
// them; else wide_lanes equal lanes sharing a queue); the others run on
// single-block lanes. The blocks are split between the two classes by their share of the
// work. Few wide lanes keep the working sets of the big systems that run at
// the same time within L2; the small systems fit beside them. The mixed
// solves give the same result on any lane, so the policy only affects speed.
struct Policy {
  int split_rows = 32768;
  int wide_lanes = 8;
};

// fewest blocks that keep a block's rows within kBlockMaxRows
int least_width(long n) {
  const long nsc = (n + kSuperRows - 1) / kSuperRows, per = kBlockMaxRows / kSuperRows;
  return (int)std::max<long>(1, (nsc + per - 1) / per);
}

// Estimated passes of a solve when no iteration count is known yet: PCG with
// a degree-k polynomial preconditioner needs ~n^(1/3) iterations on these
// 3-D pressure systems, k + 1 passes each; BiCGStab about 6 iterations of 4.
// the Chebyshev degree a pressure solve of n rows runs with
int cheb_degree_of(long n) {
  int k = 1;
  double r = 0.0;
  cheb_params(n, k, r);
  return k;
}

double model_passes(long n, bool pcg, int cheb_k) {
  return pcg ? std::max(5.0, std::cbrt((double)n)) * (std::max(cheb_k, 1) + 1) : 24.0;
}

// Lanes of one launch: their widths and classes, and per class the queue of
// systems, most work first. Classes are ordered by lane width, widest first;
// a lane takes from its own class and then from later (narrower) ones, so a
// system only ever runs on a lane at least as wide as the one planned for it.
struct LaneSet {
  std::vector<int> width, cls;
  std::vector<std::vector<int>> queue;
};

LaneSet plan_lanes(const std::vector<int>& n, const std::vector<double>& passes, const Policy& P, int cap) {
  LaneSet L;
  std::vector<std::pair<double, int>> big, small;
  double wb = 0.0, ws = 0.0;
  int need = 1;  // the widest least width among the big systems
  for (int i = 0; i < (int)n.size(); ++i) {
    const double w = passes[i] * (double)n[i];
    if (n[i] > P.split_rows || least_width(n[i]) > 1) {
      big.push_back({w, i});
      wb += w;
      need = std::max(need, least_width(n[i]));
    } else {
      small.push_back({w, i});
      ws += w;
    }
  }
  auto by_work = [](const std::pair<double, int>& x, const std::pair<double, int>& y) {
    return x.first != y.first ? x.first > y.first : x.second < y.second;
  };
  std::sort(big.begin(), big.end(), by_work);
  std::sort(small.begin(), small.end(), by_work);
  int bb = 0, bs = 0;
  if (big.empty()) {
    bs = std::min<int>(cap, (int)small.size());
  } else if (small.empty()) {
    bb = cap;
  } else {
    bs = (int)std::llround(cap * ws / (wb + ws));
    bs = std::max(1, std::min<int>(bs, std::min<int>((int)small.size(), cap - need)));
    bb = cap - bs;
  }
  if (!big.empty() && (int)big.size() <= P.wide_lanes) {
    // one lane per big system, widths in proportion to their work, so that
    // they finish the phase together (each at least its least width); each
    // lane is its own class holding exactly its system
    std::vector<int> w(big.size());
    int used = 0;
    for (size_t j = 0; j < big.size(); ++j) {
      w[j] = std::max(least_width(n[big[j].second]), (int)std::floor(bb * big[j].first / wb));
      used += w[j];
    }
    while (used > bb) {  // trim the lanes with most room above their least width
      size_t jm = 0;
      for (size_t j = 1; j < w.size(); ++j)
        if (w[j] - least_width(n[big[j].second]) > w[jm] - least_width(n[big[jm].second])) jm = j;
      if (w[jm] <= least_width(n[big[jm].second])) break;
      --w[jm];
      --used;
    }
    for (size_t j = 0; used < bb; j = (j + 1) % w.size(), ++used) ++w[j];  // spare blocks, most work first
    std::vector<size_t> ord(w.size());
    for (size_t j = 0; j < ord.size(); ++j) ord[j] = j;
    std::stable_sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return w[x] > w[y]; });
    for (size_t j : ord) {
      L.width.push_back(w[j]);
      L.cls.push_back((int)L.queue.size());
      L.queue.push_back({big[j].second});
    }
  } else if (!big.empty()) {
    // more big systems than wide lanes: equal lanes sharing one queue
    const int k = std::max(1, std::min(P.wide_lanes, bb / need));
    for (int j = 0; j < k; ++j) {
      L.width.push_back(bb / k + (j < bb % k ? 1 : 0));
      L.cls.push_back(0);
    }
    L.queue.push_back({});
    for (auto& e : big) L.queue.back().push_back(e.second);
  }
  const int sc = (int)L.queue.size();  // the single-block class
  L.queue.push_back({});
  for (auto& e : small) L.queue.back().push_back(e.second);
  for (int j = 0; j < bs; ++j) {
    L.width.push_back(1);
    L.cls.push_back(sc);
  }
  return L;
}

// done[i] for every live case, then the count of running cases and of
// cases whose bounded wait ran out.
__global__ void k_batch_flags(const BatchCase* __restrict__ cases, int n, int* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevStatus* st = cases[i].d.st;
  const int d = st->abort != 0;
  flags[i] = d;
  if (!d) atomicAdd(&flags[n], 1);
  if (st->timeout) atomicAdd(&flags[n + 1], 1);
}

// Batch tables live in stream-ordered memory on the batch's stream: freeing
// them never waits for other streams' work.
template <typename T>
int dev_alloc(T*& p, size_t n, cudaStream_t s) {
  p = nullptr;
  MGPU_CUDA(cudaMallocAsync((void**)&p, std::max<size_t>(n, 1) * sizeof(T), s));
  return 0;
}

}  // namespace

// One batched Krylov launch with its device tables.
struct BatchLaunch {
  bool pcg = false;
  int ell = 0;  // 0 CSR, 1 ELL, 2 ELL with the L2 prefetch
  LanePlan plan{};
  std::vector<void*> owned;
};

// A Krylov phase: the systems of every member case that takes part.
struct BatchPhase {
  bool pcg = false;
  int comp = 0;   // momentum component
  int icorr = -1; // pressure corrector (pcg)
  std::vector<int> mixed;  // member indices solved in batched launches
  std::vector<int> fp64;   // member indices solved one by one
  std::vector<double> passes;  // per mixed system: passes of its last solve (0: unknown)
  bool pf = false;             // the phase's systems together exceed the L2 share: prefetch
  BatchSys* d_sys = nullptr;
  std::vector<BatchLaunch> launches;
};

struct MgpuBatch {
  std::vector<MgpuCase*> cases;
  std::vector<int> gen;   // run generation of each member when prepared
  std::vector<int> live;  // members with a run begun, in table order
  cudaStream_t stream = nullptr;
  Policy policy;
  bool autotune = true;
  bool tuned = false;         // this preparation's solves were measured and re-planned
  bool policy_tuned = false;  // the autotuner has picked the policy
  // assembly tables
  BatchCase* d_cases = nullptr;
  int* d_blk[4] = {nullptr, nullptr, nullptr, nullptr};
  AsmBatch asmb{};
  int maxcorr = 1;
  std::vector<BatchPhase> phases;
  unsigned long long* d_bars = nullptr;
  double* d_part = nullptr;
  int* d_flags = nullptr;  // done[live] + running + timed out
  bool any_blend = false, any_outflow = false;
  int cap = 0;
  bool prepared = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool use_graph = true;
  int launches_per_iter = 0;
  // kernels this batch has run: counted at every launch site; a graph's
  // kernels once per replay (graph_kernels: counted while capturing, when
  // nothing runs)
  int64_t launched = 0;
  int64_t graph_kernels = 0;
  double tune_ms = 0.0, step_ms = 0.0;
  int64_t iters = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  // profiling
  bool profiling = false;
  unsigned long long* d_lane_t = nullptr;
  std::vector<cudaEvent_t> pev;
  double phase_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double asm_ms = 0.0, lane_max_ms = 0.0, lane_mean_ms = 0.0;
  int64_t profiled_iters = 0;

  void free_launch(BatchLaunch& L) {
    for (void* p : L.owned) cudaFreeAsync(p, stream);
    L.owned.clear();
  }
  void free_phases() {
    for (auto& ph : phases) {
      for (auto& L : ph.launches) free_launch(L);
      if (ph.d_sys) cudaFreeAsync(ph.d_sys, stream);
    }
    phases.clear();
  }
  void free_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  void free_tables() {
    free_graph();
    free_phases();
    if (d_cases) cudaFreeAsync(d_cases, stream);
    for (auto& p : d_blk)
      if (p) cudaFreeAsync(p, stream);
    d_cases = nullptr;
    for (auto& p : d_blk) p = nullptr;
    prepared = false;
  }
  ~MgpuBatch() {
    free_tables();
    if (d_bars) cudaFreeAsync(d_bars, stream);
    if (d_part) cudaFreeAsync(d_part, stream);
    if (d_flags) cudaFreeAsync(d_flags, stream);
    if (d_lane_t) cudaFreeAsync(d_lane_t, stream);
    for (auto e : pev) cudaEventDestroy(e);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (stream) release_stream(stream);
  }
};

namespace {

// Device tables of the launches of one phase under policy P. Passes per
// system: measured (ph.passes, from the last iteration's counts) or modelled.
int build_launches(MgpuBatch* b, BatchPhase& ph, const Policy& P) {
  for (auto& L : ph.launches) b->free_launch(L);
  ph.launches.clear();
  for (int ell = 0; ell < 2; ++ell) {
    std::vector<int> items, n;  // positions in ph.mixed
    std::vector<double> passes;
    for (int k = 0; k < (int)ph.mixed.size(); ++k) {
      const MgpuCase* c = b->cases[ph.mixed[k]];
      if ((c->d.ell_col != nullptr) == (ell == 1)) {
        items.push_back(k);
        n.push_back(c->d.N);
        passes.push_back(k < (int)ph.passes.size() && ph.passes[k] > 0
                             ? ph.passes[k]
                             : model_passes(c->d.N, ph.pcg, ph.pcg ? cheb_degree_of(c->d.N) : 1));
      }
    }
    if (items.empty()) continue;
    const int mode = ell == 1 ? (ph.pf ? 2 : 1) : 0;
    const int cap = std::max(1, batch_capacity(ph.pcg, mode) - g_batch_reserve);
    const LaneSet ls = plan_lanes(n, passes, P, cap);
    std::vector<BatchLane> hl;
    std::vector<int> block_lane, q_items, q_start;
    for (size_t j = 0; j < ls.width.size(); ++j) {
      hl.push_back(BatchLane{(int)block_lane.size(), ls.width[j], ls.cls[j], 0});
      for (int k = 0; k < ls.width[j]; ++k) block_lane.push_back((int)j);
    }
    for (const auto& q : ls.queue) {
      q_start.push_back((int)q_items.size());
      for (int i : q) q_items.push_back(items[i]);
    }
    q_start.push_back((int)q_items.size());
    const int ncls = (int)ls.queue.size();
    BatchLaunch L;
    L.pcg = ph.pcg;
    L.ell = mode;
    BatchLane* dl = nullptr;
    int *dbl = nullptr, *dqi = nullptr, *dqs = nullptr, *dqh = nullptr, *dslot = nullptr;
    TRY(dev_alloc(dl, hl.size(), b->stream));
    L.owned.push_back(dl);
    TRY(dev_alloc(dbl, block_lane.size(), b->stream));
    L.owned.push_back(dbl);
    TRY(dev_alloc(dqi, q_items.size(), b->stream));
    L.owned.push_back(dqi);
    TRY(dev_alloc(dqs, q_start.size(), b->stream));
    L.owned.push_back(dqs);
    TRY(dev_alloc(dqh, (size_t)ncls, b->stream));
    L.owned.push_back(dqh);
    TRY(dev_alloc(dslot, 2 * hl.size(), b->stream));
    L.owned.push_back(dslot);
    MGPU_CUDA(cudaMemcpyAsync(dl, hl.data(), sizeof(BatchLane) * hl.size(), cudaMemcpyHostToDevice, b->stream));
    MGPU_CUDA(cudaMemcpyAsync(dbl, block_lane.data(), sizeof(int) * block_lane.size(), cudaMemcpyHostToDevice, b->stream));
    MGPU_CUDA(cudaMemcpyAsync(dqi, q_items.data(), sizeof(int) * q_items.size(), cudaMemcpyHostToDevice, b->stream));
    MGPU_CUDA(cudaMemcpyAsync(dqs, q_start.data(), sizeof(int) * q_start.size(), cudaMemcpyHostToDevice, b->stream));
    L.plan = LanePlan{ph.d_sys, dl, dbl, dqi, dqs, dqh, dslot, b->d_bars, b->d_part, nullptr, ncls, (int)hl.size(),
                      (int)block_lane.size()};
    ph.launches.push_back(std::move(L));
  }
  return 0;
}

// one batched assembly kernel over every member, counted
int batch_op(MgpuBatch* b, int op, int arg) {
  b->launched++;
  return launch_batch_asm(op, arg, b->asmb, b->stream);
}

int run_phase(MgpuBatch* b, const BatchPhase& ph) {
  for (const auto& L : ph.launches) {
    TRY(launch_mixed_batch(L.plan, L.pcg, L.ell, b->stream));
    b->launched++;
  }
  for (int m : ph.fp64) {
    MgpuCase* c = b->cases[m];
    const bool tr = c->run_mode == 1;
    const KrylovArgs a = ph.pcg ? ppe_args(c, std::min(3 + ph.icorr, MGPU_MAXSOLVE - 1), tr) : mom_args(c, ph.comp, tr);
    const int64_t before = c->launches;
    TRY(krylov(c, a, !ph.pcg, b->stream));
    b->launched += c->launches - before;
  }
  return 0;
}

// Kernels one iteration launches.
int count_launches(const MgpuBatch* b) {
  if (b->live.empty()) return 0;
  int n = 0;
  for (const auto& ph : b->phases) {
    n += (int)ph.launches.size();
    for (int m : ph.fp64) {
      const MgpuCase* c = b->cases[m];
      const bool jac = ph.pcg ? c->ctrl.ppe_precond == MGPU_PPE_JACOBI : c->ctrl.mom_solver == MGPU_MOM_JACOBI;
      n += jac ? 1 : 2;
    }
  }
  // begin, momentum x3 (+ the interior pass, or the limiter x3), apc,
  // gradients, rhiechow, 3 per corrector, diag x2
  n += 1 + 3 + 3 + 3 * b->maxcorr + 2;
  n += b->any_blend ? 3 : 1;
  if (b->any_outflow) n += 1;
  return n;
}

int prepare(MgpuBatch* b) {
  b->free_tables();
  b->live.clear();
  for (int k = 0; k < (int)b->cases.size(); ++k) {
    b->gen[k] = b->cases[k]->run_gen;
    if (b->cases[k]->run_mode >= 0) b->live.push_back(k);
  }
  const int K = (int)b->live.size();
  std::vector<BatchCase> hc(K);
  std::vector<int> ncorr(b->cases.size(), 0);
  std::vector<int> blk[4];
  b->maxcorr = 1;
  b->any_blend = b->any_outflow = false;
  for (int j = 0; j < K; ++j) {
    const int k = b->live[j];
    MgpuCase* c = b->cases[k];
    BatchCase& B = hc[j];
    std::memset(&B, 0, sizeof(B));
    B.d = c->d;
    B.P = c->P;
    B.transient = c->run_mode;
    B.time_scheme = c->ctrl.time_scheme;
    B.has_outflow = c->has_outflow;
    B.ncorr = c->run_mode == 1 ? std::max(1, c->ctrl.n_correct) : 1;
    ncorr[k] = B.ncorr;
    b->maxcorr = std::max(b->maxcorr, std::min(B.ncorr, MGPU_MAXSOLVE - 3));
    b->any_blend = b->any_blend || c->P.conv_blend > 0.0;
    b->any_outflow = b->any_outflow || c->has_outflow;
    const long N = c->d.N, F = c->d.F;
    const long nb[4] = {(N + 255) / 256, (F + 255) / 256, (3 * N + 255) / 256, 1};
    for (int r = 0; r < 4; ++r) {
      B.blk0[r] = (int)blk[r].size();
      blk[r].insert(blk[r].end(), (size_t)nb[r], j);
    }
  }
  b->prepared = true;
  if (K == 0) return 0;
  TRY(dev_alloc(b->d_cases, K, b->stream));
  MGPU_CUDA(cudaMemcpyAsync(b->d_cases, hc.data(), sizeof(BatchCase) * K, cudaMemcpyHostToDevice, b->stream));
  b->asmb.cases = b->d_cases;
  for (int r = 0; r < 4; ++r) {
    TRY(dev_alloc(b->d_blk[r], blk[r].size(), b->stream));
    MGPU_CUDA(cudaMemcpyAsync(b->d_blk[r], blk[r].data(), sizeof(int) * blk[r].size(), cudaMemcpyHostToDevice, b->stream));
    b->asmb.blk_case[r] = b->d_blk[r];
    b->asmb.nblk[r] = (int)blk[r].size();
  }
  // Krylov phases
  for (int ph = 0; ph < 3 + b->maxcorr; ++ph) {
    BatchPhase P;
    P.pcg = ph >= 3;
    P.comp = ph < 3 ? ph : 0;
    P.icorr = ph >= 3 ? ph - 3 : -1;
    std::vector<BatchSys> hs;
    for (int k : b->live) {
      MgpuCase* c = b->cases[k];
      if (P.pcg && P.icorr >= ncorr[k]) continue;
      if (c->ctrl.precision != MGPU_PREC_MIXED) {
        P.fp64.push_back(k);
        continue;
      }
      const bool tr = c->run_mode == 1;
      BatchSys s;
      std::memset(&s, 0, sizeof(s));
      s.a = P.pcg ? ppe_args(c, std::min(3 + P.icorr, MGPU_MAXSOLVE - 1), tr) : mom_args(c, P.comp, tr);
      s.a.precond = 1;
      s.m = mixed_args(c, !P.pcg);
      hs.push_back(s);
      P.mixed.push_back(k);
    }
    // the systems of a phase run side by side: together larger than the L2
    // share, every system prefetches
    double rows_bytes = 0.0;
    for (size_t q = 0; q < hs.size(); ++q) rows_bytes += (double)hs[q].a.n * mixed_row_bytes(hs[q].m.ell_w);
    P.pf = rows_bytes > g_prefetch_mb * 1048576.0;
    for (auto& h : hs) h.m.pf = (h.m.ell_col && P.pf) ? 1 : 0;
    if (!hs.empty()) {
      TRY(dev_alloc(P.d_sys, hs.size(), b->stream));
      MGPU_CUDA(cudaMemcpyAsync(P.d_sys, hs.data(), sizeof(BatchSys) * hs.size(), cudaMemcpyHostToDevice, b->stream));
    }
    b->phases.push_back(std::move(P));
    TRY(build_launches(b, b->phases.back(), b->policy));
  }
  b->launches_per_iter = count_launches(b);
  b->tuned = false;  // the first step measures the solves and re-plans
  return 0;
}

// Krylov iteration counts of the iteration in progress, per live case and solve slot
__global__ void k_gather_its(const BatchCase* __restrict__ cases, int n, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DeviceCase& d = cases[i].d;
  const MgpuIterRec* rec = d.recs + d.st->cur_it;
  for (int k = 0; k < MGPU_MAXSOLVE; ++k) out[i * MGPU_MAXSOLVE + k] = rec->lin_it[k];
}

// Passes of every mixed system's last solve, from the records of the
// iteration in progress: inner iterations times the passes of one iteration
// (PCG: the fused SpMV pass plus the k - 1 Chebyshev passes and the update;
// BiCGStab: two SpMV and the updates), plus the prologue and true residuals.
int measure_passes(MgpuBatch* b) {
  const int K = (int)b->live.size();
  if (K == 0) return 0;
  int* d_its = nullptr;
  TRY(dev_alloc(d_its, (size_t)K * MGPU_MAXSOLVE, b->stream));
  k_gather_its<<<(K + 127) / 128, 128, 0, b->stream>>>(b->d_cases, K, d_its);
  b->launched++;
  std::vector<int> its((size_t)K * MGPU_MAXSOLVE);
  cudaError_t e = cudaMemcpyAsync(its.data(), d_its, sizeof(int) * its.size(), cudaMemcpyDeviceToHost, b->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
  cudaFreeAsync(d_its, b->stream);
  if (e != cudaSuccess) return cuda_fail(e, "iteration counts", __FILE__, __LINE__);
  std::vector<int> live_of(b->cases.size(), -1);
  for (int j = 0; j < K; ++j) live_of[b->live[j]] = j;
  for (auto& ph : b->phases) {
    const int slot = ph.pcg ? std::min(3 + ph.icorr, MGPU_MAXSOLVE - 1) : ph.comp;
    ph.passes.assign(ph.mixed.size(), 0.0);
    for (size_t k = 0; k < ph.mixed.size(); ++k) {
      const long n = b->cases[ph.mixed[k]]->d.N;
      const double per = ph.pcg ? (double)(std::max(cheb_degree_of(n), 1) + 1) : 4.0;
      ph.passes[k] = 3.0 + per * std::max(0, its[(size_t)live_of[ph.mixed[k]] * MGPU_MAXSOLVE + slot]);
    }
  }
  return 0;
}

// One iteration launch by launch with events around every phase and lane
// timestamps in the first pressure phase; accumulates into the batch's
// The momentum assembly of component comp for every member: with any member
// on the limited convection scheme, each component whole (after the previous
// component's solve); else the boundary faces, sources and relaxation after
// the one interior pass (BOP_MOM_INTERIOR) of the iteration.
int momentum_assembly(MgpuBatch* b, int comp) {
  if (b->any_blend) {
    TRY(batch_op(b, BOP_LIMITER, comp));
    return batch_op(b, BOP_MOMENTUM, comp);
  }
  return batch_op(b, BOP_MOM_FINISH, comp);
}

// profile.
int profiled_iteration(MgpuBatch* b) {
  cudaStream_t s = b->stream;
  if (!b->d_lane_t) TRY(dev_alloc(b->d_lane_t, 2 * (size_t)b->cap, b->stream));
  while (b->pev.size() < 32) {
    cudaEvent_t e;
    MGPU_CUDA(cudaEventCreate(&e));
    b->pev.push_back(e);
  }
  int ne = 0;
  auto mark = [&]() { cudaEventRecord(b->pev[ne++], s); };
  std::vector<int> kind;  // per interval: -1 assembly, else the phase index
  mark();
  TRY(batch_op(b, BOP_BEGIN_ITER, 0));
  if (!b->any_blend) TRY(batch_op(b, BOP_MOM_INTERIOR, 0));
  for (int comp = 0; comp < 3; ++comp) {
    TRY(momentum_assembly(b, comp));
    mark();
    kind.push_back(-1);
    TRY(run_phase(b, b->phases[comp]));
    mark();
    kind.push_back(comp);
  }
  TRY(batch_op(b, BOP_APC, 0));
  TRY(batch_op(b, BOP_GRADIENTS, 0));
  TRY(batch_op(b, BOP_RHIECHOW, 0));
  if (b->any_outflow) TRY(batch_op(b, BOP_OUTFLOW, 0));
  std::vector<LanePlan> saved;
  for (int ic = 0; ic < b->maxcorr; ++ic) {
    TRY(batch_op(b, BOP_PPE, ic));
    mark();
    kind.push_back(-1);
    BatchPhase& ph = b->phases[3 + ic];
    if (ic == 0 && !ph.launches.empty()) ph.launches[0].plan.lane_t = b->d_lane_t;
    const int rc = run_phase(b, ph);
    if (ic == 0 && !ph.launches.empty()) ph.launches[0].plan.lane_t = nullptr;
    TRY(rc);
    mark();
    kind.push_back(3 + ic);
    TRY(batch_op(b, BOP_CORRECT_CELLS, ic));
    TRY(batch_op(b, BOP_CORRECT_FLUX, ic));
  }
  TRY(batch_op(b, BOP_DIAG, 0));
  TRY(batch_op(b, BOP_DIAG_FINALIZE, 0));
  mark();
  kind.push_back(-1);
  MGPU_CUDA(cudaStreamSynchronize(s));
  for (int k = 0; k + 1 < ne; ++k) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, b->pev[k], b->pev[k + 1]);
    if (kind[k] < 0)
      b->asm_ms += ms;
    else if (kind[k] < 8)
      b->phase_ms[kind[k]] += ms;
  }
  if (b->phases.size() > 3 && !b->phases[3].launches.empty()) {
    const LanePlan& P = b->phases[3].launches[0].plan;
    std::vector<unsigned long long> t(2 * (size_t)P.nlanes);
    TRY(copy_sync(t.data(), b->d_lane_t, sizeof(unsigned long long) * t.size(), cudaMemcpyDeviceToHost, b->stream));
    double mx = 0.0, sum = 0.0;
    for (int l = 0; l < P.nlanes; ++l) {
      const double ms = (double)(t[2 * l + 1] - t[2 * l]) * 1e-6;
      mx = std::max(mx, ms);
      sum += ms;
    }
    b->lane_max_ms += mx;
    b->lane_mean_ms += P.nlanes ? sum / P.nlanes : 0.0;
  }
  b->profiled_iters++;
  return 0;
}

// One outer iteration / time step of every member.
int enqueue_iteration(MgpuBatch* b, bool tune) {
  cudaStream_t s = b->stream;
  TRY(batch_op(b, BOP_BEGIN_ITER, 0));
  if (!b->any_blend) TRY(batch_op(b, BOP_MOM_INTERIOR, 0));
  for (int comp = 0; comp < 3; ++comp) {
    TRY(momentum_assembly(b, comp));
    TRY(run_phase(b, b->phases[comp]));
  }
  TRY(batch_op(b, BOP_APC, 0));
  TRY(batch_op(b, BOP_GRADIENTS, 0));
  TRY(batch_op(b, BOP_RHIECHOW, 0));
  if (b->any_outflow) TRY(batch_op(b, BOP_OUTFLOW, 0));
  for (int ic = 0; ic < b->maxcorr; ++ic) {
    TRY(batch_op(b, BOP_PPE, ic));
    BatchPhase& ph = b->phases[3 + ic];
    if (tune && ic == 0) {
      // Run the first pressure solve on the modelled plan, then re-plan every
      // phase on the measured iteration counts under each candidate policy
      // and time the pressure solve again: it starts from pp = 0 and leaves
      // its inputs alone, and its result does not depend on the plan, so
      // every trial solves the same systems to the same result.
      cudaEvent_t a0, a1;
      MGPU_CUDA(cudaEventCreate(&a0));
      MGPU_CUDA(cudaEventCreate(&a1));
      MGPU_CUDA(cudaEventRecord(a0, s));
      TRY(run_phase(b, ph));
      MGPU_CUDA(cudaEventRecord(a1, s));
      TRY(measure_passes(b));
      float total = 0.f;
      MGPU_CUDA(cudaEventElapsedTime(&total, a0, a1));
      if (b->autotune && !b->policy_tuned && !ph.mixed.empty()) {
        static const int splits[] = {8192, 32768};
        static const int wides[] = {2, 4, 8, 16};
        float best = 1e30f;
        Policy bp = b->policy;
        for (int sr : splits)
          for (int wl : wides) {
            const Policy cand{sr, wl};
            TRY(build_launches(b, ph, cand));
            MGPU_CUDA(cudaEventRecord(a0, s));
            TRY(run_phase(b, ph));
            MGPU_CUDA(cudaEventRecord(a1, s));
            MGPU_CUDA(cudaEventSynchronize(a1));
            float ms = 0.f;
            MGPU_CUDA(cudaEventElapsedTime(&ms, a0, a1));
            total += ms;
            if (ms < best) {
              best = ms;
              bp = cand;
            }
          }
        b->policy = bp;
        b->policy_tuned = true;
      }
      cudaEventDestroy(a0);
      cudaEventDestroy(a1);
      b->tune_ms += total;
      b->tuned = true;
      for (auto& p : b->phases) TRY(build_launches(b, p, b->policy));
      b->launches_per_iter = count_launches(b);
      TRY(batch_op(b, BOP_CORRECT_CELLS, ic));
      TRY(batch_op(b, BOP_CORRECT_FLUX, ic));
      continue;
    }
    TRY(run_phase(b, ph));
    TRY(batch_op(b, BOP_CORRECT_CELLS, ic));
    TRY(batch_op(b, BOP_CORRECT_FLUX, ic));
  }
  TRY(batch_op(b, BOP_DIAG, 0));
  TRY(batch_op(b, BOP_DIAG_FINALIZE, 0));
  return 0;
}

int capture(MgpuBatch* b) {
  b->free_graph();
  cudaStream_t s = b->stream;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    b->use_graph = false;
    return 0;
  }
  const int64_t before = b->launched;
  const int rc = enqueue_iteration(b, false);
  b->graph_kernels = b->launched - before;  // recorded, not run
  b->launched = before;
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(s, &g);
  if (rc != 0 || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    b->use_graph = false;  // replay the launches one by one instead
    return rc;
  }
  if (cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    b->exec = nullptr;
    b->use_graph = false;
    return 0;
  }
  b->graph = g;
  return 0;
}

bool stale(const MgpuBatch* b) {
  for (size_t k = 0; k < b->cases.size(); ++k)
    if (b->gen[k] != b->cases[k]->run_gen) return true;
  return false;
}

}  // namespace

extern "C" {

int mgpu_case_begin(MgpuCase* c, int mode, int nsteps, int* ier) {
  if (!c || !ier || (mode != 0 && mode != 1)) {
    set_error("mgpu_case_begin: invalid argument");
    return MGPU_E_ARG;
  }
  *ier = 0;
  c->run_mode = -1;
  c->P.pimple = 0;
  int n;
  if (mode == 1) {
    if (!c->ctrl.transient) {
      *ier = 30;
      return 0;
    }
    if (c->ctrl.dt <= 0.0) {
      *ier = 31;
      return 0;
    }
    n = std::max(1, c->ctrl.n_time_max);
  } else {
    n = c->ctrl.outer_max;
  }
  if (nsteps > 0) n = std::min(n, nsteps);
  n = std::max(n, 0);
  TRY(ensure_recs(c, n + 1));
  TRY(reset_status(c, mode, n + 1));
  if (n == 0) {  // nothing to run: the case starts finished
    const int one = 1;
    MGPU_CUDA(cudaMemcpyAsync(&c->d.st->abort, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
  }
  TRY(launch_fill(c->d.apc, c->d.N, 1.0, c->stream));
  TRY(launch_gradients(c->d, c->P, c->stream));
  if (mode == 1) TRY(launch_rhiechow(c->d, c->P, c->stream));
  MGPU_CUDA(cudaStreamSynchronize(c->stream));
  c->run_mode = mode;
  c->run_gen++;
  return 0;
}

int mgpu_case_finish(MgpuCase* c, MgpuIterRec* log, int logcap, int* nrec, int* ier) {
  if (!c || !ier) return MGPU_E_ARG;
  DevStatus h{};
  MGPU_CUDA(cudaMemcpyAsync(&h, c->d.st, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  MGPU_CUDA(cudaStreamSynchronize(c->stream));
  if (nrec) *nrec = h.cur_it;
  *ier = h.ier;
  if (log && logcap > 0 && h.cur_it > 0)
    TRY(copy_sync(log, c->d.recs, sizeof(MgpuIterRec) * (size_t)std::min(h.cur_it, logcap), cudaMemcpyDeviceToHost,
                  c->stream));
  if (h.timeout) {
    set_error("a bounded device wait ran out (grid barrier)");
    return MGPU_E_TIMEOUT;
  }
  return 0;
}

int mgpu_batch_create(MgpuCase* const* cases, int ncases, MgpuBatch** out) {
  if (!cases || ncases <= 0 || !out) {
    set_error("mgpu_batch_create: invalid argument");
    return MGPU_E_ARG;
  }
  *out = nullptr;
  for (int k = 0; k < ncases; ++k)
    for (int j = 0; j < k; ++j)
      if (!cases[k] || cases[k] == cases[j]) {
        set_error("mgpu_batch_create: null or repeated case");
        return MGPU_E_ARG;
      }
  for (int k = 0; k < ncases; ++k)
    if (cases[k]->d.energy) {
      set_error("mgpu_batch_create: cases with the energy equation are stepped one by one (mgpu_simple_run ...)");
      return MGPU_E_ARG;
    }
  MgpuBatch* b = new MgpuBatch();
  b->cases.assign(cases, cases + ncases);
  b->gen.assign(ncases, -1);
  auto fail = [&](int e) {
    delete b;
    return e;
  };
  b->stream = acquire_stream();
  if (!b->stream) {
    set_error("cudaStreamCreate failed");
    return fail(MGPU_E_CUDA);
  }
  b->cap = 1;
  for (int ell = 0; ell < 3; ++ell)
    b->cap = std::max(b->cap, std::max(batch_capacity(true, ell), batch_capacity(false, ell)));
  if (int e = dev_alloc(b->d_bars, b->cap, b->stream)) return fail(e);
  if (int e = dev_alloc(b->d_part, 8l * b->cap, b->stream)) return fail(e);
  if (int e = dev_alloc(b->d_flags, ncases + 2, b->stream)) return fail(e);
  if (cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess) {
    set_error("cudaEventCreate failed");
    return fail(MGPU_E_CUDA);
  }
  *out = b;
  return 0;
}

int mgpu_batch_destroy(MgpuBatch* b) {
  delete b;
  return 0;
}

int mgpu_batch_set_policy(MgpuBatch* b, int split_rows, int wide_lanes) {
  if (!b || split_rows < 0 || wide_lanes < 0 || ((split_rows == 0) != (wide_lanes == 0)) ||
      split_rows > kBlockMaxRows) {
    set_error("mgpu_batch_set_policy: invalid argument");
    return MGPU_E_ARG;
  }
  b->autotune = split_rows == 0;
  b->policy_tuned = false;
  if (!b->autotune) b->policy = Policy{split_rows, wide_lanes};
  b->prepared = false;
  return 0;
}

int mgpu_batch_step(MgpuBatch* b, int iters, int* active) {
  if (!b || iters < 0) {
    set_error("mgpu_batch_step: invalid argument");
    return MGPU_E_ARG;
  }
  if (!b->prepared || stale(b)) TRY(prepare(b));
  const int K = (int)b->live.size();
  if (K == 0) {
    if (active) *active = 0;
    return 0;
  }
  MGPU_CUDA(cudaEventRecord(b->e0, b->stream));
  for (int it = 0; it < iters; ++it) {
    if (!b->tuned) {  // first iteration: measure the solves, re-plan (and autotune)
      TRY(enqueue_iteration(b, true));
      b->free_graph();
    } else if (b->profiling) {
      TRY(profiled_iteration(b));
    } else if (b->use_graph) {
      if (!b->exec) TRY(capture(b));
      if (b->exec) {
        MGPU_CUDA(cudaGraphLaunch(b->exec, b->stream));
        b->launched += b->graph_kernels;
      } else {
        TRY(enqueue_iteration(b, false));
      }
    } else {
      TRY(enqueue_iteration(b, false));
    }
    b->iters++;
  }
  MGPU_CUDA(cudaMemsetAsync(b->d_flags + K, 0, 2 * sizeof(int), b->stream));
  k_batch_flags<<<(K + 127) / 128, 128, 0, b->stream>>>(b->d_cases, K, b->d_flags);
  MGPU_LAUNCH_CHECK("k_batch_flags");
  b->launched++;
  int cnt[2] = {0, 0};
  MGPU_CUDA(cudaMemcpyAsync(cnt, b->d_flags + K, sizeof(cnt), cudaMemcpyDeviceToHost, b->stream));
  MGPU_CUDA(cudaEventRecord(b->e1, b->stream));
  MGPU_CUDA(cudaStreamSynchronize(b->stream));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, b->e0, b->e1);
  b->step_ms += ms;
  if (active) *active = cnt[0];
  if (cnt[1]) {
    set_error("a bounded device wait ran out (grid barrier) in a batched case");
    return MGPU_E_TIMEOUT;
  }
  return 0;
}

int mgpu_batch_poll(MgpuBatch* b, int* done) {
  if (!b || !done) return MGPU_E_ARG;
  if (!b->prepared || stale(b)) TRY(prepare(b));
  for (size_t k = 0; k < b->cases.size(); ++k) done[k] = 1;  // members without a run count as done
  const int K = (int)b->live.size();
  if (K == 0) return 0;
  std::vector<int> h(K);
  MGPU_CUDA(cudaMemsetAsync(b->d_flags + K, 0, 2 * sizeof(int), b->stream));
  k_batch_flags<<<(K + 127) / 128, 128, 0, b->stream>>>(b->d_cases, K, b->d_flags);
  MGPU_LAUNCH_CHECK("k_batch_flags");
  b->launched++;
  MGPU_CUDA(cudaMemcpyAsync(h.data(), b->d_flags, sizeof(int) * K, cudaMemcpyDeviceToHost, b->stream));
  MGPU_CUDA(cudaStreamSynchronize(b->stream));
  for (int j = 0; j < K; ++j) done[b->live[j]] = h[j];
  return 0;
}

int mgpu_batch_run(MgpuBatch* b, const int* mode, int nsteps, int* nrec, int* ier) {
  if (!b || !mode || !ier) return MGPU_E_ARG;
  const int K = (int)b->cases.size();
  int it_max = 0;
  std::vector<int> live;
  for (int k = 0; k < K; ++k) {
    MgpuCase* c = b->cases[k];
    TRY(mgpu_case_begin(c, mode[k], nsteps, &ier[k]));
    if (nrec) nrec[k] = 0;
    if (c->run_mode < 0) continue;  // rejected (ier 30 / 31): not run, as mgpu_piso_run
    live.push_back(k);
    const int n = mode[k] == 1 ? std::max(1, c->ctrl.n_time_max) : c->ctrl.outer_max;
    it_max = std::max(it_max, nsteps > 0 ? std::min(n, nsteps) : n);
  }
  int done_it = 0;
  while (done_it < it_max) {
    const int chunk = std::min(32, it_max - done_it);
    int active = 0;
    TRY(mgpu_batch_step(b, chunk, &active));
    done_it += chunk;
    if (active == 0) break;
  }
  for (int k : live) {
    int nr = 0, e = 0;
    TRY(mgpu_case_finish(b->cases[k], nullptr, 0, &nr, &e));
    if (nrec) nrec[k] = nr;
    ier[k] = e;
  }
  return 0;
}

int mgpu_batch_plan(int nsys, const int* rows, const double* passes, int split_rows, int wide_lanes, int capacity,
                    int* sys_class, int* lane_width, int* nlanes) {
  if (nsys < 0 || (nsys > 0 && !rows) || split_rows <= 0 || split_rows > kBlockMaxRows || wide_lanes <= 0 ||
      capacity <= 0 || !nlanes) {
    set_error("mgpu_batch_plan: invalid argument");
    return MGPU_E_ARG;
  }
  const std::vector<int> n(rows, rows + nsys);
  std::vector<double> ps(nsys);
  for (int i = 0; i < nsys; ++i) ps[i] = passes ? passes[i] : model_passes(n[i], true, cheb_degree_of(n[i]));
  const LaneSet L = plan_lanes(n, ps, Policy{split_rows, wide_lanes}, capacity);
  for (size_t c = 0; c < L.queue.size(); ++c)
    for (int i : L.queue[c])
      if (sys_class) sys_class[i] = (int)c;
  for (size_t j = 0; j < L.width.size(); ++j)
    if (lane_width) lane_width[j] = L.width[j];
  *nlanes = (int)L.width.size();
  return 0;
}

int mgpu_batch_set_profiling(MgpuBatch* b, int on) {
  if (!b) return MGPU_E_ARG;
  b->profiling = on != 0;
  return 0;
}

int mgpu_batch_info(const MgpuBatch* b, MgpuBatchInfo* info) {
  if (!b || !info) return MGPU_E_ARG;
  MgpuBatchInfo r{};
  r.ncases = (int)b->cases.size();
  r.split_rows = b->policy.split_rows;
  r.wide_lanes = b->policy.wide_lanes;
  r.autotuned = b->policy_tuned ? 1 : 0;
  r.graph = b->exec ? 1 : 0;
  r.launches_per_iter = b->launches_per_iter;
  r.gpu_launches = b->launched;
  if (b->phases.size() > 3)
    for (const auto& L : b->phases[3].launches) {
      r.lanes += L.plan.nlanes;
      r.blocks = std::max(r.blocks, L.plan.nblocks);
    }
  r.tune_ms = b->tune_ms;
  r.step_ms = b->step_ms;
  r.iters = b->iters;
  for (int k = 0; k < 8; ++k) r.phase_ms[k] = b->phase_ms[k];
  r.asm_ms = b->asm_ms;
  r.lane_max_ms = b->lane_max_ms;
  r.lane_mean_ms = b->lane_mean_ms;
  r.profiled_iters = b->profiled_iters;
  *info = r;
  return 0;
}

}  // extern "C"
