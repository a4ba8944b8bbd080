// The request server: resident fields, cached models, continuous batching.
//
// The reference answers one planning problem per build_model + spvi_2 run
// (src/Makefile:1-24).  Served here, a request names a resident field, a
// heading set, a target and a start cell.  Its transitions do not depend on
// the target, so one base model per (field, heading set) is built once, with
// no terminal cells and with each row's reward sum kept, and a request only
// re-targets R near its target and solves:
//
//  * rows whose samples land in the target (not through an obstacle, whose
//    reward is replaced by r_outbound, src/build_model.cu:538-540) get
//    r_terminal instead of the late-time penalty (:343-354) for each such
//    sample: sum + count * (r_terminal - late), divided by nrzns as the
//    builder does (:567).  For integer-valued rewards (the "time" reward with
//    integer dt, r_outbound, r_terminal) every partial sum is exact and R is
//    bit-identical to a model built with the target; otherwise it differs by
//    the rounding of the reward sums.
//  * the target's own rows are terminal: the reference leaves such a sample
//    in place with reward 0 (:523-545); the batched sweep evaluates that row.
//
// A worker thread drains the queue: requests whose base model is resident
// join the next batch at once; a missing model is built (one per iteration)
// when the HBM budget admits it, after evicting idle models least recently
// used.  A batch is one persistent launch of the batched sweep (graph
// replay).  Latency is measured from submission to completion.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "internal.h"

#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

namespace e2e {
namespace {

// R of the rows of cells [wi0, wi0+wh) x [wj0, wj0+ww), layers 0..nt-2, for a
// target subgrid [ti, ti+tsg) x [tj, tj+tsg), from a base model built without
// terminal cells; layout [t][wi][wj][a].
template <typename PtrT, typename CntT>
__global__ void k_retarget(ViModel M, DevProblem P, const int32_t* __restrict__ mask,
                           const float* __restrict__ sumR, int ti, int tj, int tsg, int wi0, int wj0,
                           int wh, int ww, float* __restrict__ Rwin) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int na = P.na;
  const int64_t total = (int64_t)(P.nt - 1) * wh * ww * na;
  if (idx >= total) return;
  const int a = (int)(idx % na);
  int64_t q = idx / na;
  const int wj = (int)(q % ww);
  q /= ww;
  const int wi = (int)(q % wh);
  const int t = (int)(q / wh);
  const int g = P.g, i = wi0 + wi, j = wj0 + wj;
  const int64_t nc = (int64_t)g * g;
  const int64_t cell = (int64_t)i * g + j;
  const int64_t row = ((int64_t)t * nc + cell) * na + a;
  float sum = sumR[row];
  const bool term1 = i >= ti && i < ti + tsg && j >= tj && j < tj + tsg;
  if (term1) {
    Rwin[idx] = 0.f;  // terminal row: evaluated by the sweep itself
    return;
  }
  if (__ldg(mask + (int64_t)t * nc + cell) != 1) {  // S1 in an obstacle: no move (:541-543)
    const bool late = t > P.nt - 20;
    float r_nt = 0.f;
    if (late) r_nt += 0.05 * P.r_out;
    const float delta = P.r_term - r_nt;
    const PtrT* rp = reinterpret_cast<const PtrT*>(M.row_ptr);
    const CntT* cnt = reinterpret_cast<const CntT*>(M.cnt);
    const int64_t b = (int64_t)rp[row], e = (int64_t)rp[row + 1];
    const int64_t base = (int64_t)(t + 1) * nc;
    for (int64_t k = b; k < e; ++k) {
      const int64_t c2 = (int64_t)M.col[k] - base;
      const int i2 = (int)(c2 / g), j2 = (int)(c2 - (int64_t)(c2 / g) * g);
      if (i2 >= ti && i2 < ti + tsg && j2 >= tj && j2 < tj + tsg && !through_obstacle(P, mask, t, i, j, i2, j2))
        sum += (float)cnt[k] * delta;
    }
  }
  Rwin[idx] = sum / P.nrzns;
}

// value and action at each request's start state
__global__ void k_gather_starts(const uint64_t* __restrict__ tab, int n, float* out_v, int32_t* out_a) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const float* V = reinterpret_cast<const float*>(tab[3 * k]);
  const int32_t* pi = reinterpret_cast<const int32_t*>(tab[3 * k + 1]);
  const int64_t s = (int64_t)tab[3 * k + 2];
  out_v[k] = V[s];
  out_a[k] = pi[s];
}

using Clock = std::chrono::steady_clock;

struct Field {
  e2e_problem prob{};
  DevFields F{};
  std::vector<void*> owned;
  int64_t bytes = 0;
};

struct ModelEntry {
  int fid = 0, angles = 0;
  e2e_model* m = nullptr;
  DevProblem D{};
  std::vector<void*> owned;  // D's device tables
  int64_t bytes = 0;
  uint64_t last_used = 0;
};

struct Req {
  int64_t id = 0;
  e2e_request r{};
  Clock::time_point submit;
  double queue_ms = 0;
  float* V = nullptr;
  int32_t* pi = nullptr;
  float* Rwin = nullptr;
  int64_t bytes = 0;
  e2e_result res{};
};

}  // namespace

// models above this many states are solved in launches of their own
constexpr int64_t kLargeStates = 4000000;

struct Server {
  e2e_server_opts opts{};
  int device = 0;
  int64_t budget = 0;
  std::atomic<int64_t> used{0};
  std::vector<Field*> fields;
  std::map<std::pair<int, int>, ModelEntry*> models;
  std::mutex mu;
  std::condition_variable cv, cv_done;
  std::deque<Req*> pending;
  std::deque<e2e_result> done;
  std::map<int64_t, Req*> kept;
  std::thread worker;
  bool stop = false;
  int64_t next_id = 1;
  uint64_t tick = 0;
  cudaStream_t st = nullptr;
  // statistics
  int64_t n_done = 0, n_batches = 0, n_builds = 0, n_evicted = 0, n_failed = 0;
  double build_ms = 0, solve_ms = 0;
  int max_batch_seen = 0;
  // per-batch scratch
  uint64_t* h_tab = nullptr;
  float* h_v = nullptr;
  int32_t* h_a = nullptr;
  uint64_t* d_tab = nullptr;
  float* d_v = nullptr;
  int32_t* d_a = nullptr;
  int cap = 0;

  e2e_status init_scratch(int n) {
    if (n <= cap) return E2E_OK;
    if (h_tab) {
      cudaFreeHost(h_tab);
      cudaFreeHost(h_v);
      cudaFreeHost(h_a);
      cudaFree(d_tab);
      cudaFree(d_v);
      cudaFree(d_a);
    }
    cap = std::max(n, 256);
    CK(cudaHostAlloc((void**)&h_tab, sizeof(uint64_t) * 3 * cap, cudaHostAllocDefault));
    CK(cudaHostAlloc((void**)&h_v, sizeof(float) * cap, cudaHostAllocDefault));
    CK(cudaHostAlloc((void**)&h_a, sizeof(int32_t) * cap, cudaHostAllocDefault));
    CK(cudaMalloc((void**)&d_tab, sizeof(uint64_t) * 3 * cap));
    CK(cudaMalloc((void**)&d_v, sizeof(float) * cap));
    CK(cudaMalloc((void**)&d_a, sizeof(int32_t) * cap));
    return E2E_OK;
  }

  static int64_t estimate_model_bytes(const e2e_problem& p, int angles) {
    const int64_t rows = (int64_t)(p.nt - 1) * p.gsize * p.gsize * angles * p.num_ac_speeds;
    // CSR (row_ptr, R, reward sums, ~3.5 entries of 6 bytes) and the sliced copy
    return rows * 80 + ((int64_t)1 << 20);
  }

  void free_model(ModelEntry* me) {
    used -= me->bytes;
    e2e_model_free(me->m);
    for (void* p : me->owned) dfree(p, st);
    delete me;
  }

  // evict idle models, least recently used first, until `need` fits
  bool make_room(int64_t need, const std::vector<std::pair<int, int>>& busy) {
    while (used + need > budget) {
      ModelEntry* victim = nullptr;
      std::pair<int, int> vkey;
      for (auto& kv : models) {
        if (std::find(busy.begin(), busy.end(), kv.first) != busy.end()) continue;
        if (!victim || kv.second->last_used < victim->last_used) {
          victim = kv.second;
          vkey = kv.first;
        }
      }
      if (!victim) return false;
      models.erase(vkey);
      free_model(victim);
      ++n_evicted;
    }
    return true;
  }

  e2e_status build_model_for(int fid, int angles, ModelEntry** out) {
    const Field* f = fields[fid];
    e2e_problem p = f->prob;
    p.num_ac_angles = angles;
    p.num_actions = angles * p.num_ac_speeds;
    p.term_subgrid_size = 0;  // base model: no terminal cells
    e2e_fields ef{f->F.u, f->F.v, f->F.ui, f->F.vi, f->F.Y, f->F.s, f->F.mask};
    e2e_build_opts bo{};
    bo.count_type = E2E_COUNT_AUTO;
    bo.keep_reward_parts = 1;
    auto t0 = Clock::now();
    e2e_model* m = nullptr;
    e2e_status s = e2e_build_model(&p, &ef, E2E_DEVICE, &bo, &m, st);
    if (s != E2E_OK) return s;
    double pms = 0;
    s = ensure_pack(m, &pms, st);
    if (s != E2E_OK) {
      e2e_model_free(m);
      return s;
    }
    auto* me = new ModelEntry();
    me->fid = fid;
    me->angles = angles;
    me->m = m;
    DeviceScratch keep(st);
    s = make_dev_problem(&p, st, &me->D, &keep);
    me->owned = keep.ptrs;
    keep.ptrs.clear();
    if (s != E2E_OK) {
      free_model(me);
      return s;
    }
    me->bytes = model_bytes(m) + (m->pack ? m->pack->bytes : 0) + (m->sumR ? m->ns * m->na * 4 : 0);
    used += me->bytes;
    build_ms += std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    ++n_builds;
    *out = me;
    return E2E_OK;
  }

  void finish(Req* q, int status) {
    q->res.request_id = q->id;
    q->res.tag = q->r.tag;
    q->res.status = status;
    q->res.latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - q->submit).count();
    q->res.queue_ms = q->queue_ms;
    if (status != E2E_OK) ++n_failed;
    std::lock_guard<std::mutex> lk(mu);
    done.push_back(q->res);
    ++n_done;
    if (q->r.keep_outputs && status == E2E_OK) {
      kept[q->id] = q;
    } else {
      release(q);
      delete q;
    }
    cv_done.notify_all();
  }

  void release(Req* q) {
    dfree(q->V, st);
    dfree(q->pi, st);
    dfree(q->Rwin, st);
    q->V = nullptr;
    q->pi = nullptr;
    q->Rwin = nullptr;
    used -= q->bytes;
    q->bytes = 0;
  }

  void loop() {
    cudaSetDevice(device);
    while (true) {
      std::vector<Req*> batch;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stop || !pending.empty(); });
        if (stop && pending.empty()) return;
        while (!pending.empty() && (int)batch.size() < opts.max_batch) {
          batch.push_back(pending.front());
          pending.pop_front();
        }
      }
      const auto t_take = Clock::now();
      for (Req* q : batch) q->queue_ms = std::chrono::duration<double, std::milli>(t_take - q->submit).count();
      // models: resident ones are used now; at most one missing model is built
      std::vector<std::pair<int, int>> busy;
      for (Req* q : batch) busy.push_back({q->r.field_id, q->r.num_ac_angles});
      std::vector<Req*> ready, later;
      bool built = false;
      for (Req* q : batch) {
        const auto key = std::make_pair(q->r.field_id, q->r.num_ac_angles);
        auto it = models.find(key);
        if (it == models.end() && !built) {
          const int64_t need = estimate_model_bytes(fields[key.first]->prob, key.second);
          if (!make_room(need, busy)) {
            // models of this batch free up once it completes; with none, it never fits
            bool other_busy = false;
            for (const auto& b : busy)
              if (b != key && models.count(b)) other_busy = true;
            if (other_busy) later.push_back(q);
            else finish(q, E2E_ERR_NOMEM);
            continue;
          }
          ModelEntry* me = nullptr;
          e2e_status s = build_model_for(key.first, key.second, &me);
          built = true;
          if (s != E2E_OK) {
            finish(q, s);
            continue;
          }
          it = models.emplace(key, me).first;
        }
        if (it == models.end()) {
          later.push_back(q);
          continue;
        }
        it->second->last_used = ++tick;
        ready.push_back(q);
      }
      // per-request outputs and re-targeted R (admission by the budget)
      std::vector<BatchJobSpec> jobs;
      std::vector<Req*> run;
      for (Req* q : ready) {
        ModelEntry* me = models[{q->r.field_id, q->r.num_ac_angles}];
        const e2e_model* m = me->m;
        const int g = m->prob.gsize, del = (m->prob.neighb_gsize - 1) / 2, tsg = 1;
        const int ti = q->r.i_term, tj = q->r.j_term;
        const int wi0 = std::max(0, ti - del), wi1 = std::min(g, ti + tsg + del);
        const int wj0 = std::max(0, tj - del), wj1 = std::min(g, tj + tsg + del);
        const int64_t nwin = (int64_t)(m->nt - 1) * (wi1 - wi0) * (wj1 - wj0) * m->na;
        const int64_t need = m->ns * 8 + nwin * 4;
        if (used + need > budget && !make_room(need, busy)) {
          if (run.empty()) finish(q, E2E_ERR_NOMEM);  // nothing in flight will free memory
          else later.push_back(q);
          continue;
        }
        if (dalloc((void**)&q->V, sizeof(float) * m->ns, st) != cudaSuccess ||
            dalloc((void**)&q->pi, sizeof(int32_t) * m->ns, st) != cudaSuccess ||
            dalloc((void**)&q->Rwin, sizeof(float) * std::max<int64_t>(nwin, 1), st) != cudaSuccess) {
          cudaGetLastError();
          release(q);
          later.push_back(q);
          continue;
        }
        q->bytes = need;
        used += need;
        const ViModel M = vi_model(m);
        const unsigned blocks = (unsigned)((nwin + 255) / 256);
        cudaError_t e = cudaSuccess;
        if (nwin > 0) {
          if (m->index_bits == 32)
            k_retarget<int32_t, uint16_t><<<blocks, 256, 0, st>>>(M, me->D, fields[me->fid]->F.mask, m->sumR, ti, tj,
                                                                  tsg, wi0, wj0, wi1 - wi0, wj1 - wj0, q->Rwin);
          else
            k_retarget<int64_t, uint16_t><<<blocks, 256, 0, st>>>(M, me->D, fields[me->fid]->F.mask, m->sumR, ti, tj,
                                                                  tsg, wi0, wj0, wi1 - wi0, wj1 - wj0, q->Rwin);
          e = cudaGetLastError();
        }
        if (e != cudaSuccess) {
          release(q);
          finish(q, E2E_ERR_CUDA);
          continue;
        }
        BatchJobSpec js;
        js.m = m;
        js.V = q->V;
        js.pi = q->pi;
        js.Rwin = q->Rwin;
        js.ti = ti;
        js.tj = tj;
        js.tsg = tsg;
        js.wi0 = wi0;
        js.wj0 = wj0;
        js.wh = wi1 - wi0;
        js.ww = wj1 - wj0;
        jobs.push_back(js);
        run.push_back(q);
      }
      // one launch per group: requests on large models (more than
      // kLargeStates states) after the others, so that a batch of small
      // requests never waits for a large model's solve in the same launch
      auto run_group = [&](std::vector<BatchJobSpec>& jobs, std::vector<Req*>& run) {
        if (run.empty()) return;
        BatchResult br;
        // the heuristic schedule unless one is given: no timing runs in the request path
        e2e_status s = solve_batch(jobs, opts.schedule ? opts.schedule : 0x400, st, &br);
        solve_ms += br.seconds * 1e3;
        ++n_batches;
        max_batch_seen = std::max(max_batch_seen, (int)run.size());
        if (s == E2E_OK) s = init_scratch((int)run.size());
        if (s == E2E_OK) {
          for (size_t k = 0; k < run.size(); ++k) {
            const e2e_model* m = jobs[k].m;
            h_tab[3 * k] = reinterpret_cast<uint64_t>(run[k]->V);
            h_tab[3 * k + 1] = reinterpret_cast<uint64_t>(run[k]->pi);
            h_tab[3 * k + 2] = (uint64_t)((int64_t)run[k]->r.i_start * m->prob.gsize + run[k]->r.j_start);
          }
          const int n = (int)run.size();
          cudaError_t e = cudaMemcpyAsync(d_tab, h_tab, sizeof(uint64_t) * 3 * n, cudaMemcpyHostToDevice, st);
          if (e == cudaSuccess) {
            k_gather_starts<<<(n + 127) / 128, 128, 0, st>>>(d_tab, n, d_v, d_a);
            e = cudaGetLastError();
          }
          if (e == cudaSuccess) e = cudaMemcpyAsync(h_v, d_v, sizeof(float) * n, cudaMemcpyDeviceToHost, st);
          if (e == cudaSuccess) e = cudaMemcpyAsync(h_a, d_a, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st);
          if (e == cudaSuccess) e = cudaStreamSynchronize(st);
          if (e != cudaSuccess) s = cuda_fail(e, "gather");
        }
        for (size_t k = 0; k < run.size(); ++k) {
          Req* q = run[k];
          q->res.batch_size = (int32_t)run.size();
          if (s == E2E_OK) {
            q->res.value_at_start = h_v[k];
            q->res.action_at_start = h_a[k];
          }
          finish(q, s);
        }
      };
      std::vector<BatchJobSpec> jobs_large;
      std::vector<Req*> run_large;
      {
        size_t w = 0;
        for (size_t k = 0; k < run.size(); ++k) {
          if (jobs[k].m->ns > kLargeStates) {
            jobs_large.push_back(jobs[k]);
            run_large.push_back(run[k]);
          } else {
            jobs[w] = jobs[k];
            run[w] = run[k];
            ++w;
          }
        }
        jobs.resize(w);
        run.resize(w);
      }
      run_group(jobs, run);
      run_group(jobs_large, run_large);
      if (!later.empty()) {
        std::lock_guard<std::mutex> lk(mu);
        for (auto it = later.rbegin(); it != later.rend(); ++it) pending.push_front(*it);
      }
    }
  }
};

}  // namespace e2e

using e2e::Server;

extern "C" e2e_status e2e_server_create(const e2e_server_opts* opts, e2e_server** out) {
  using namespace e2e;
  if (!out) return fail(E2E_ERR_INVALID, "null output handle");
  *out = nullptr;
  auto* S = new Server();
  if (opts) S->opts = *opts;
  if (S->opts.max_batch <= 0) S->opts.max_batch = 256;
  if (S->opts.max_batch > 1024) S->opts.max_batch = 1024;
  CK(cudaGetDevice(&S->device));
  size_t fr = 0, tot = 0;
  CK(cudaMemGetInfo(&fr, &tot));
  S->budget = S->opts.hbm_budget > 0 ? S->opts.hbm_budget : (int64_t)(fr * 0.8);
  CK(cudaStreamCreateWithFlags(&S->st, cudaStreamNonBlocking));
  S->worker = std::thread([S] { S->loop(); });
  *out = reinterpret_cast<e2e_server*>(S);
  return E2E_OK;
}

extern "C" e2e_status e2e_server_add_field(e2e_server* srv, const e2e_problem* p, const e2e_fields* f,
                                           int where, int32_t* field_id) {
  using namespace e2e;
  auto* S = reinterpret_cast<Server*>(srv);
  if (!S || !p || !f || !field_id) return fail(E2E_ERR_INVALID, "null argument");
  e2e_status vs = validate_problem(p);
  if (vs != E2E_OK) return vs;
  if (where != E2E_HOST && where != E2E_DEVICE) return fail(E2E_ERR_INVALID, "bad fields_where");
  auto* fl = new Field();
  fl->prob = *p;
  const size_t nc = (size_t)p->gsize * p->gsize, nt = (size_t)p->nt, nm = (size_t)p->nmodes;
  const size_t b2 = sizeof(float) * nt * nc, bm = sizeof(float) * nt * nm * nc;
  const size_t by = sizeof(float) * nt * (size_t)p->nrzns * nm;
  const void* src[7] = {f->u, f->v, f->ui, f->vi, f->yi, f->s, f->mask};
  const size_t bytes[7] = {b2, b2, bm, bm, by, b2, sizeof(int32_t) * nt * nc};
  void* dst[7] = {nullptr};
  for (int k = 0; k < 7; ++k) {
    if (!src[k] || bytes[k] == 0) continue;
    cudaError_t e = cudaMalloc(&dst[k], bytes[k]);
    if (e == cudaSuccess)
      e = cudaMemcpy(dst[k], src[k], bytes[k], where == E2E_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) {
      for (void* d : dst)
        if (d) cudaFree(d);
      delete fl;
      return cuda_fail(e, "e2e_server_add_field");
    }
    fl->owned.push_back(dst[k]);
    fl->bytes += (int64_t)bytes[k];
  }
  fl->F.u = (const float*)dst[0];
  fl->F.v = (const float*)dst[1];
  fl->F.ui = (const float*)dst[2];
  fl->F.vi = (const float*)dst[3];
  fl->F.Y = (const float*)dst[4];
  fl->F.s = (const float*)dst[5];
  fl->F.mask = (const int32_t*)dst[6];
  std::lock_guard<std::mutex> lk(S->mu);
  *field_id = (int32_t)S->fields.size();
  S->fields.push_back(fl);
  return E2E_OK;
}

extern "C" e2e_status e2e_server_submit(e2e_server* srv, const e2e_request* r, int64_t* request_id) {
  using namespace e2e;
  auto* S = reinterpret_cast<Server*>(srv);
  if (!S || !r) return fail(E2E_ERR_INVALID, "null argument");
  auto* q = new Req();
  q->submit = Clock::now();
  q->r = *r;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (r->field_id < 0 || r->field_id >= (int32_t)S->fields.size()) {
      delete q;
      return fail(E2E_ERR_INVALID, "unknown field_id");
    }
    const e2e_problem& p = S->fields[r->field_id]->prob;
    const int g = p.gsize;
    if (r->num_ac_angles < 1 || r->num_ac_angles * p.num_ac_speeds > 32 || r->i_term < 0 || r->i_term >= g ||
        r->j_term < 0 || r->j_term >= g || r->i_start < 0 || r->i_start >= g || r->j_start < 0 || r->j_start >= g) {
      delete q;
      return fail(E2E_ERR_INVALID, "request outside the field's grid or heading limits");
    }
    q->id = S->next_id++;
    if (request_id) *request_id = q->id;
    S->pending.push_back(q);
  }
  S->cv.notify_one();
  return E2E_OK;
}

extern "C" e2e_status e2e_server_cancel(e2e_server* srv, int64_t request_id) {
  using namespace e2e;
  auto* S = reinterpret_cast<Server*>(srv);
  if (!S) return fail(E2E_ERR_INVALID, "null server");
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (auto it = S->pending.begin(); it != S->pending.end(); ++it) {
      Req* q = *it;
      if (q->id != request_id) continue;
      // still queued: it holds no device memory (outputs are allocated when a
      // batch takes it), so it leaves the queue with its result at once
      S->pending.erase(it);
      q->res.request_id = q->id;
      q->res.tag = q->r.tag;
      q->res.status = E2E_ERR_CANCELLED;
      q->res.latency_ms = std::chrono::duration<double, std::milli>(Clock::now() - q->submit).count();
      q->res.queue_ms = q->res.latency_ms;
      S->done.push_back(q->res);
      ++S->n_done;
      ++S->n_failed;
      delete q;
      S->cv_done.notify_all();
      return E2E_OK;
    }
    if (request_id <= 0 || request_id >= S->next_id) return fail(E2E_ERR_INVALID, "unknown request id");
  }
  return fail(E2E_ERR_BUSY, "request already taken into a batch or finished; it completes normally");
}

extern "C" e2e_status e2e_server_poll(e2e_server* srv, e2e_result* out, int32_t max, int32_t* n_out,
                                      double wait_s) {
  using namespace e2e;
  auto* S = reinterpret_cast<Server*>(srv);
  if (!S || !n_out || (max > 0 && !out)) return fail(E2E_ERR_INVALID, "null argument");
  std::unique_lock<std::mutex> lk(S->mu);
  if (S->done.empty() && wait_s > 0)
    S->cv_done.wait_for(lk, std::chrono::duration<double>(wait_s), [&] { return !S->done.empty(); });
  int n = 0;
  while (n < max && !S->done.empty()) {
    out[n++] = S->done.front();
    S->done.pop_front();
  }
  *n_out = n;
  return E2E_OK;
}

extern "C" e2e_status e2e_server_fetch(e2e_server* srv, int64_t request_id, float* value_out,
                                       int32_t* policy_out, int out_where) {
  using namespace e2e;
  auto* S = reinterpret_cast<Server*>(srv);
  if (!S) return fail(E2E_ERR_INVALID, "null server");
  Req* q = nullptr;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->kept.find(request_id);
    if (it == S->kept.end()) return fail(E2E_ERR_INVALID, "no kept outputs for this request");
    q = it->second;
    S->kept.erase(it);
  }
  const e2e_problem& p = S->fields[q->r.field_id]->prob;
  const int64_t ns = (int64_t)p.gsize * p.gsize * p.nt;
  const cudaMemcpyKind k = out_where == E2E_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  cudaError_t e = cudaSuccess;
  if (value_out) e = cudaMemcpy(value_out, q->V, sizeof(float) * ns, k);
  if (e == cudaSuccess && policy_out) e = cudaMemcpy(policy_out, q->pi, sizeof(int32_t) * ns, k);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->release(q);
  }
  cudaStreamSynchronize(S->st);
  delete q;
  if (e != cudaSuccess) return cuda_fail(e, "e2e_server_fetch");
  return E2E_OK;
}

extern "C" e2e_status e2e_server_get_stats(e2e_server* srv, e2e_server_stats* out) {
  using namespace e2e;
  auto* S = reinterpret_cast<Server*>(srv);
  if (!S || !out) return fail(E2E_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  std::memset(out, 0, sizeof(*out));
  out->completed = S->n_done;
  out->failed = S->n_failed;
  out->pending = (int64_t)S->pending.size();
  out->batches = S->n_batches;
  out->models_built = S->n_builds;
  out->models_evicted = S->n_evicted;
  out->models_resident = (int64_t)S->models.size();
  out->max_batch = S->max_batch_seen;
  out->bytes_in_use = S->used;
  out->budget_bytes = S->budget;
  out->build_ms = S->build_ms;
  out->solve_ms = S->solve_ms;
  return E2E_OK;
}

extern "C" e2e_status e2e_server_destroy(e2e_server* srv) {
  using namespace e2e;
  auto* S = reinterpret_cast<Server*>(srv);
  if (!S) return E2E_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv.notify_all();
  if (S->worker.joinable()) S->worker.join();
  cudaStreamSynchronize(S->st);
  for (auto& kv : S->kept) {
    S->release(kv.second);
    delete kv.second;
  }
  for (auto& kv : S->models) S->free_model(kv.second);
  for (Field* f : S->fields) {
    for (void* p : f->owned) cudaFree(p);
    delete f;
  }
  cudaStreamSynchronize(S->st);
  if (S->h_tab) {
    cudaFreeHost(S->h_tab);
    cudaFreeHost(S->h_v);
    cudaFreeHost(S->h_a);
    cudaFree(S->d_tab);
    cudaFree(S->d_v);
    cudaFree(S->d_a);
  }
  cudaStreamDestroy(S->st);
  delete S;
  return E2E_OK;
}
