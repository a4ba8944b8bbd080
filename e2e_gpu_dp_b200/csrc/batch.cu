// Batched layered solves: many models, or many re-targeted requests on shared
// models, solved in one persistent cooperative launch (k_vi_batch) that is
// captured once in a CUDA graph and replayed for every later batch of the
// same launch shape.  The reference solves one model per process
// (src/spvi_2.cu:730-795); batching has no counterpart there.
//
// The device job table has a fixed capacity, so the graph's nodes never
// change: a copy of the pinned host table into the device table, a reset of
// the error word and of the per-(job, layer) completion counters, and the
// kernel.  A new batch rewrites the pinned
// host table and replays the graph.  The schedule (warps per chunk, kernel
// variant and L2 prefetch) is picked per batch shape by timing the 16
// candidates on the first batch of that shape.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "internal.h"

#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

namespace e2e {
namespace {

constexpr int kJobCap = kViBatchJobCap;
constexpr int kLayerCap = 4096;

struct Choice {
  int groups = 1, tune = VI_TUNE_PF_NEXT;
};

class BatchSolver {
 public:
  std::mutex mu;
  int device = -1;
  void* d_table = nullptr;
  unsigned char* h_table = nullptr;
  unsigned int* d_sync = nullptr;  // [1]: error bits of the bounded waits
  int* d_done = nullptr;           // [kJobCap][kLayerCap] chunks finished per (job, layer)
  cudaStream_t priv = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr, t0 = nullptr, t1 = nullptr;
  std::map<std::tuple<int, int, int, int, int>, cudaGraphExec_t> graphs;  // mode, cnt, G, tune, grid
  std::map<std::tuple<int, int, int, int>, Choice> tuned;                // mode, cnt, log2 jobs, log2 items
  size_t table_bytes = vi_batch_table_bytes(kJobCap, kLayerCap);
  size_t done_bytes = sizeof(int) * (size_t)kJobCap * kLayerCap;

  e2e_status init(int dev) {
    if (device == dev) return E2E_OK;
    if (device >= 0) return fail(E2E_ERR_UNSUPPORTED, "batch solver bound to another device");
    CK(dalloc(&d_table, table_bytes, nullptr));
    CK(dalloc((void**)&d_sync, sizeof(unsigned int) * 2, nullptr));
    CK(dalloc((void**)&d_done, done_bytes, nullptr));
    CK(cudaHostAlloc((void**)&h_table, table_bytes, cudaHostAllocDefault));
    std::memset(h_table, 0, table_bytes);
    CK(cudaStreamCreateWithFlags(&priv, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ev_in, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&ev_out, cudaEventDisableTiming));
    CK(cudaEventCreate(&t0));
    CK(cudaEventCreate(&t1));
    CK(cudaStreamSynchronize(nullptr));
    device = dev;
    return E2E_OK;
  }

  // the batch's kernel, in stream order on `st`
  e2e_status run(int mode, int cnt, const Choice& ch, int grid, bool use_graph, cudaStream_t st,
                 bool* graphed) {
    *graphed = false;
    if (use_graph) {
      auto key = std::make_tuple(mode, cnt, ch.groups, ch.tune, grid);
      auto it = graphs.find(key);
      if (it == graphs.end()) {
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        CK(cudaStreamBeginCapture(priv, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaMemcpyAsync(d_table, h_table, table_bytes, cudaMemcpyHostToDevice, priv);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_sync, 0, sizeof(unsigned int) * 2, priv);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_done, 0, done_bytes, priv);
        if (e == cudaSuccess)
          e = launch_vi_batch(d_table, kJobCap, kLayerCap, mode, cnt, ch.groups, grid, ch.tune, d_done, d_sync + 1,
                              priv);
        cudaError_t e2 = cudaStreamEndCapture(priv, &g);
        if (e == cudaSuccess && e2 == cudaSuccess) e = cudaGraphInstantiate(&ge, g, 0);
        if (g) cudaGraphDestroy(g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
          cudaGetLastError();
          use_graph = false;  // capture refused: launch directly
        } else {
          it = graphs.emplace(key, ge).first;
        }
      }
      if (use_graph) {
        CK(cudaEventRecord(ev_in, st));
        CK(cudaStreamWaitEvent(priv, ev_in, 0));
        CK(cudaGraphLaunch(it->second, priv));
        CK(cudaEventRecord(ev_out, priv));
        CK(cudaStreamWaitEvent(st, ev_out, 0));
        *graphed = true;
        return E2E_OK;
      }
    }
    CK(cudaMemcpyAsync(d_table, h_table, table_bytes, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(d_sync, 0, sizeof(unsigned int) * 2, st));
    CK(cudaMemsetAsync(d_done, 0, done_bytes, st));
    CK(launch_vi_batch(d_table, kJobCap, kLayerCap, mode, cnt, ch.groups, grid, ch.tune, d_done, d_sync + 1, st));
    return E2E_OK;
  }

  e2e_status check_sync(cudaStream_t st) {
    unsigned int h[2] = {0, 0};
    CK(cudaMemcpyAsync(h, d_sync, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h[1]) return fail(E2E_ERR_DEVICE, "a bounded wait of the batched sweep gave up");
    return E2E_OK;
  }
};

BatchSolver& solver() {
  static BatchSolver* s = new BatchSolver();  // lives until exit (graphs hold device memory)
  return *s;
}

int ilog2(int64_t v) {
  int r = 0;
  while (v > 1) {
    v >>= 1;
    ++r;
  }
  return r;
}

}  // namespace

e2e_status solve_batch(const std::vector<BatchJobSpec>& jobs, int schedule, cudaStream_t st,
                       BatchResult* res) {
  *res = BatchResult{};
  if (jobs.empty()) return E2E_OK;
  const int gsel = schedule & 15;
  if ((schedule & ~0x77f) || (gsel != 0 && gsel != 1 && gsel != 2 && gsel != 4 && gsel != 8))
    return fail(E2E_ERR_INVALID, "schedule: bits 0-3 warps per chunk (0, 1, 2, 4, 8), bits 4-6 tuning, "
                                 "bit 8 tuning given, bit 9 no CUDA graph, bit 10 heuristic schedule");
  const bool tune_given = (schedule & 0x100) != 0;
  const bool heuristic = (schedule & 0x400) != 0;
  const bool use_graph = (schedule & 0x200) == 0;
  for (const auto& j : jobs) {
    if (!j.m || !j.V || !j.pi) return fail(E2E_ERR_INVALID, "batch job without model or outputs");
    if (!j.m->layered || j.m->nt < 2) return fail(E2E_ERR_UNSUPPORTED, "batched solves need time-layered models");
  }
  int dev = 0;
  CK(cudaGetDevice(&dev));
  BatchSolver& S = solver();
  std::lock_guard<std::mutex> lock(S.mu);
  e2e_status s = S.init(dev);
  if (s != E2E_OK) return s;
  for (const auto& j : jobs) {
    double ms = 0;
    s = ensure_pack(j.m, &ms, st);
    if (s != E2E_OK) return s;
    res->pack_ms += ms;
  }
  // launches: one per (layout, count type) group and per kJobCap jobs
  std::map<std::pair<int, int>, std::vector<int>> groups;
  for (int i = 0; i < (int)jobs.size(); ++i) {
    const ViPack& P = jobs[i].m->pack->v;
    if (P.nlayers > kLayerCap) return fail(E2E_ERR_UNSUPPORTED, "batched solve: more than 4096 layers");
    if (jobs[i].Rwin && P.g <= 0) return fail(E2E_ERR_UNSUPPORTED, "re-targeted job without grid geometry");
    groups[{P.ent_mode, P.count_type}].push_back(i);
  }
  CK(cudaEventRecord(S.t0, st));
  for (auto& kv : groups) {
    std::vector<int>& idx = kv.second;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
      return jobs[a].m->pack->v.nlayers > jobs[b].m->pack->v.nlayers;
    });
    for (size_t off = 0; off < idx.size(); off += kJobCap) {
      const int n = (int)std::min<size_t>(kJobCap, idx.size() - off);
      unsigned char* h = S.h_table;
      auto* H = reinterpret_cast<ViBatchHeader*>(h);
      auto* J = reinterpret_cast<ViJob*>(h + kViBatchJobsOffset);
      int* cum = reinterpret_cast<int*>(J + kJobCap);
      int* nact = cum + kJobCap + 1;
      int maxL = 0, min_na = 1 << 30;
      int64_t total = 0;
      double step_bytes = 0;  // one layer of every job
      cum[0] = 0;
      for (int q = 0; q < n; ++q) {
        const BatchJobSpec& js = jobs[idx[off + q]];
        const ViPack& P = js.m->pack->v;
        ViJob& jb = J[q];
        jb.P = P;
        jb.V = js.V;
        jb.pi = js.pi;
        jb.Rwin = js.Rwin;
        jb.ti = js.ti;
        jb.tj = js.tj;
        jb.tsg = js.tsg;
        jb.wi0 = js.wi0;
        jb.wj0 = js.wj0;
        jb.wh = js.wh;
        jb.ww = js.ww;
        total += P.cpl;
        if (total >= (int64_t)1 << 30) return fail(E2E_ERR_UNSUPPORTED, "batched solve: too many chunks per layer");
        cum[q + 1] = (int)total;
        maxL = std::max(maxL, P.nlayers);
        min_na = std::min(min_na, P.na);
        res->stream_bytes += pack_sweep_bytes(P);
        step_bytes += (double)pack_sweep_bytes(P) / P.nlayers;
      }
      for (int k = 0; k < maxL; ++k) {
        int a = 0;
        while (a < n && J[a].P.nlayers > k) ++a;
        nact[k] = a;
      }
      H->njobs = n;
      H->max_layers = maxL;
      const int mode = kv.first.first, cnt = kv.first.second;
      // CTAs: enough for the widest step, rounded up to a power of two so that
      // batches of similar size share one captured graph (a new launch shape
      // costs a capture and an instantiation; surplus CTAs find no items)
      auto grid_for = [&](const Choice& c) {
        const int cap = vi_batch_capacity(mode, cnt, c.tune);
        const int64_t need = (total + (8 / c.groups) - 1) / (8 / c.groups);
        int64_t q = 1;
        while (q < need) q <<= 1;
        return (int)std::max<int64_t>(1, std::min<int64_t>(cap, q));
      };
      Choice ch;
      if (tune_given) {
        ch.tune = (schedule >> 4) & 7;
        ch.groups = gsel;
      } else if (heuristic) {
        // no timing runs (request paths): prefetch the next layer while a step's
        // data fits well inside L2, and the lean kernel (with rows of exact slot
        // count it beat the look-ahead one on every served shape measured: one
        // 300x300x150 job 3.84 against 4.44 ms, four small jobs 1.02 against
        // 1.68 ms, one small job 0.87 against 0.90 ms)
        ch.tune = (step_bytes < 48e6 ? VI_TUNE_PF_NEXT : 0) | VI_TUNE_LEAN;
        ch.groups = gsel;
      } else {
        const auto key = std::make_tuple(mode, cnt, ilog2(n), ilog2(total / std::max(1, n) + 1));
        auto it = S.tuned.find(key);
        if (it != S.tuned.end()) {
          ch = it->second;
        } else {
          // time every candidate on this batch (each run fully rewrites the outputs)
          auto tt0 = std::chrono::steady_clock::now();
          float best = 1e30f;
          for (int G : {1, 2, 4, 8}) {
            if (G > min_na) continue;
            // with and without the L2 prefetch of the next layer: it pays while
            // a step's data fits L2 and costs bandwidth (evicted, read twice)
            // when it does not
            for (int tn : {(int)VI_TUNE_PF_NEXT, (int)(VI_TUNE_PF_NEXT | VI_TUNE_LEAN), 0, (int)VI_TUNE_LEAN}) {
              Choice c{G, tn};
              bool gr = false;
              cudaEvent_t a, b;
              CK(cudaEventCreate(&a));
              CK(cudaEventCreate(&b));
              CK(cudaEventRecord(a, st));
              s = S.run(mode, cnt, c, grid_for(c), false, st, &gr);
              CK(cudaEventRecord(b, st));
              CK(cudaEventSynchronize(b));
              float ms = 0;
              cudaEventElapsedTime(&ms, a, b);
              cudaEventDestroy(a);
              cudaEventDestroy(b);
              if (s != E2E_OK) return s;
              s = S.check_sync(st);
              if (s != E2E_OK) return s;
              if (ms < best) {
                best = ms;
                ch = c;
              }
            }
          }
          S.tuned[key] = ch;
          res->tune_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tt0).count();
        }
        if (ch.groups == 0) ch.groups = 1;
      }
      if (ch.groups == 0) {  // auto: split actions while that adds warps
        const int cap = vi_batch_capacity(mode, cnt, ch.tune);
        ch.groups = 1;
        while (ch.groups < 8 && ch.groups * 2 <= min_na && total * ch.groups * 2 <= (int64_t)cap * 8)
          ch.groups *= 2;
      }
      if (ch.groups > min_na) return fail(E2E_ERR_INVALID, "schedule: more warps per chunk than actions");
      const int grid = grid_for(ch);
      bool graphed = false;
      s = S.run(mode, cnt, ch, grid, use_graph, st, &graphed);
      if (s != E2E_OK) return s;
      s = S.check_sync(st);  // the pinned table is reused by the next launch
      if (s != E2E_OK) return s;
      res->launches += 1;
      res->groups = ch.groups;
      res->tune = ch.tune;
      res->grid = grid;
      res->graph = graphed ? 1 : 0;
    }
  }
  CK(cudaEventRecord(S.t1, st));
  CK(cudaEventSynchronize(S.t1));
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, S.t0, S.t1));
  res->seconds = ms * 1e-3;
  return E2E_OK;
}

}  // namespace e2e

extern "C" e2e_status e2e_spvi_solve_batch(const e2e_model* const* models, int32_t n,
                                           const e2e_vi_opts* opts, float* const* value_dev,
                                           int32_t* const* policy_dev, e2e_batch_stats* stats,
                                           void* stream) {
  using namespace e2e;
  if (n < 0 || (n > 0 && (!models || !value_dev || !policy_dev)))
    return fail(E2E_ERR_INVALID, "null batch arrays");
  if (opts && opts->method != 1) return fail(E2E_ERR_UNSUPPORTED, "batched solves use the layered method");
  std::vector<BatchJobSpec> jobs((size_t)n);
  for (int i = 0; i < n; ++i) {
    jobs[i].m = models[i];
    jobs[i].V = value_dev[i];
    jobs[i].pi = policy_dev[i];
  }
  BatchResult r;
  e2e_status s = solve_batch(jobs, opts ? opts->schedule : 0, (cudaStream_t)stream, &r);
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->jobs = n;
    stats->launches = r.launches;
    stats->groups = r.groups;
    stats->tune = r.tune;
    stats->grid = r.grid;
    stats->graph = r.graph;
    stats->seconds = r.seconds;
    stats->pack_ms = r.pack_ms;
    stats->tune_ms = r.tune_ms;
    stats->stream_bytes = r.stream_bytes;
  }
  return s;
}

// Many builds at once: each of `workers` host threads builds its share of the
// problems with e2e_build_model on its own stream, so the builder launches of
// small problems overlap on the device instead of leaving it idle between
// launches and host synchronisations.
extern "C" e2e_status e2e_build_models(const e2e_problem* problems, const e2e_fields* fields, int32_t n,
                                       int fields_where, const e2e_build_opts* opts, int32_t workers,
                                       e2e_model** out) {
  using namespace e2e;
  if (n < 0 || (n > 0 && (!problems || !fields || !out))) return fail(E2E_ERR_INVALID, "null batch arrays");
  for (int i = 0; i < n; ++i) out[i] = nullptr;
  if (n == 0) return E2E_OK;
  if (workers <= 0) workers = 4;
  workers = std::min(workers, n);
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::vector<e2e_status> st((size_t)n, E2E_OK);
  std::vector<std::string> err((size_t)n);
  std::atomic<int> next{0};
  std::vector<std::thread> th;
  for (int w = 0; w < workers; ++w) {
    th.emplace_back([&, w]() {
      (void)w;
      cudaSetDevice(dev);
      cudaStream_t s = nullptr;
      if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) s = nullptr;
      for (int i = next++; i < n; i = next++) {
        st[i] = e2e_build_model(&problems[i], &fields[i], fields_where, opts, &out[i], s);
        if (st[i] != E2E_OK) err[i] = e2e_last_error();
      }
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    });
  }
  for (auto& t : th) t.join();
  for (int i = 0; i < n; ++i) {
    if (st[i] != E2E_OK) {
      for (int k = 0; k < n; ++k) {
        e2e_model_free(out[k]);
        out[k] = nullptr;
      }
      return fail(st[i], "build " + std::to_string(i) + ": " + err[i]);
    }
  }
  return E2E_OK;
}
