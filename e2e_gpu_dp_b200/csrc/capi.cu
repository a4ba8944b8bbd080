// Host orchestration and the C ABI declared in include/e2e_dp.h.
#include <cuda_runtime.h>
#include <sys/resource.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "e2e_dp.h"
#include "internal.h"
#include "kernels.h"
#include "npy_io.h"

using namespace e2e;

// ---------------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------------
static thread_local std::string g_err;

namespace e2e {
e2e_status fail(e2e_status st, const std::string& msg) {
  g_err = msg;
  return st;
}
e2e_status cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? E2E_ERR_NOMEM : E2E_ERR_CUDA;
}
}  // namespace e2e

#define CK(call)                                          \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) return cuda_fail(_e, #call);   \
  } while (0)

// ---------------------------------------------------------------------------------
// device memory: one stream-ordered pool per device owned by the library.  Its
// release threshold is unbounded, so memory freed by one build is reused by the
// next without returning to the driver at every synchronisation (which made
// repeated builds pay for re-mapping gigabytes); e2e_memory_trim releases it.
// ---------------------------------------------------------------------------------
namespace {
std::mutex g_pool_mu;
cudaMemPool_t g_pool[64] = {};
}  // namespace

namespace e2e {
cudaError_t device_pool(cudaMemPool_t* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t thr = UINT64_MAX;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    if (e != cudaSuccess) return e;
    g_pool[dev] = pool;
  }
  *out = g_pool[dev];
  return cudaSuccess;
}

}  // namespace e2e

// ---------------------------------------------------------------------------------
// large-block cache.  Blocks of 8 MiB and more that the library frees are kept,
// with an event recorded on the freeing stream, and handed to the next request
// of about the same size (at most a quarter larger) after a stream wait on that
// event.  Repeated builds and solves then take no pool allocation at all: the
// pool serves them from its reserve too, but a request that its free ranges do
// not fit as they lie goes through the driver, which on a busy machine took from
// a few to several hundred milliseconds.  Bounded per device (a quarter of its
// memory, oldest blocks returned first); a failed pool allocation empties it and
// retries; e2e_memory_trim empties it.
// ---------------------------------------------------------------------------------
namespace {
constexpr size_t kCacheMinBytes = size_t(8) << 20;

struct CachedBlock {
  void* p;
  size_t bytes;
  cudaEvent_t ev;  // recorded on the freeing stream
  uint64_t seq;
};

struct BlockCache {
  std::mutex mu;
  std::vector<CachedBlock> free;
  std::vector<cudaEvent_t> spare_events;
  size_t free_bytes = 0, cap = 0;
  uint64_t seq = 0;
};
BlockCache g_cache[64];
// large blocks handed out, of every device (device pointers are unique): size and device
std::mutex g_live_mu;
std::unordered_map<void*, std::pair<size_t, int>> g_live;

int current_device() {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return -1;
  return dev;
}

// every cached block of the device, released on stream st once its free is done
void drop_cached(int dev, cudaStream_t st) {
  BlockCache& c = g_cache[dev];
  std::vector<CachedBlock> v;
  {
    std::lock_guard<std::mutex> lk(c.mu);
    v.swap(c.free);
    c.free_bytes = 0;
  }
  for (CachedBlock& b : v) {
    cudaStreamWaitEvent(st, b.ev, 0);
    cudaEventDestroy(b.ev);
    cudaFreeAsync(b.p, st);
  }
}
}  // namespace

namespace e2e {
cudaError_t dalloc(void** p, size_t bytes, cudaStream_t st) {
  cudaMemPool_t pool;
  cudaError_t e = device_pool(&pool);
  if (e != cudaSuccess) return e;
  if (bytes < kCacheMinBytes) return cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, st);
  const int dev = current_device();
  if (dev < 0) return cudaErrorInvalidDevice;
  BlockCache& c = g_cache[dev];
  CachedBlock got{nullptr, 0, nullptr, 0};
  {
    std::lock_guard<std::mutex> lk(c.mu);
    int best = -1;
    for (int i = 0; i < (int)c.free.size(); ++i) {
      const CachedBlock& b = c.free[i];
      if (b.bytes < bytes || b.bytes > bytes + bytes / 4) continue;
      if (best < 0 || b.bytes < c.free[best].bytes ||
          (b.bytes == c.free[best].bytes && b.seq > c.free[best].seq))
        best = i;
    }
    if (best >= 0) {
      got = c.free[best];
      c.free.erase(c.free.begin() + best);
      c.free_bytes -= got.bytes;
    }
  }
  if (got.p) {
    {
      std::lock_guard<std::mutex> lk(g_live_mu);
      g_live[got.p] = {got.bytes, dev};
    }
    e = cudaStreamWaitEvent(st, got.ev, 0);
    {
      std::lock_guard<std::mutex> lk(c.mu);
      c.spare_events.push_back(got.ev);
    }
    if (e != cudaSuccess) {
      dfree(got.p, st);
      return e;
    }
    *p = got.p;
    return cudaSuccess;
  }
  e = cudaMallocFromPoolAsync(p, bytes, pool, st);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    drop_cached(dev, st);
    e = cudaMallocFromPoolAsync(p, bytes, pool, st);
  }
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_live_mu);
  g_live[*p] = {bytes, dev};
  return cudaSuccess;
}

void dfree(void* p, cudaStream_t st) {
  if (!p) return;
  const int dev = current_device();
  size_t bytes = 0;
  {
    std::lock_guard<std::mutex> lk(g_live_mu);
    auto it = g_live.find(p);
    if (it != g_live.end()) {
      if (it->second.second == dev) bytes = it->second.first;
      g_live.erase(it);
    }
  }
  if (!bytes) {  // a small block, or one freed with another device current: to the pool
    cudaFreeAsync(p, st);
    return;
  }
  BlockCache* c = &g_cache[dev];
  cudaEvent_t ev = nullptr;
  {
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->spare_events.empty()) {
      ev = c->spare_events.back();
      c->spare_events.pop_back();
    }
  }
  if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) ev = nullptr;
  if (!ev || cudaEventRecord(ev, st) != cudaSuccess) {
    if (ev) cudaEventDestroy(ev);
    cudaFreeAsync(p, st);
    return;
  }
  std::vector<CachedBlock> evict;
  {
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->cap) {
      size_t fr = 0, total = 0;
      c->cap = cudaMemGetInfo(&fr, &total) == cudaSuccess ? total / 4 : (size_t(16) << 30);
    }
    c->free.push_back({p, bytes, ev, ++c->seq});
    c->free_bytes += bytes;
    while (c->free_bytes > c->cap && !c->free.empty()) {
      auto old = std::min_element(c->free.begin(), c->free.end(),
                                  [](const CachedBlock& a, const CachedBlock& b) { return a.seq < b.seq; });
      c->free_bytes -= old->bytes;
      evict.push_back(*old);
      c->free.erase(old);
    }
  }
  for (CachedBlock& b : evict) {
    cudaStreamWaitEvent(st, b.ev, 0);
    cudaEventDestroy(b.ev);
    cudaFreeAsync(b.p, st);
  }
}

// A stream synchronisation spins the calling thread for the whole wait (0.44 s
// of CPU per 200x200x120 build); a blocking-sync event lets it sleep and be
// woken by the device, so a busy host does not hold up the next launch.
cudaError_t sleep_sync(cudaStream_t st) {
  cudaEvent_t ev;
  cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventBlockingSync | cudaEventDisableTiming);
  if (e != cudaSuccess) return e;
  e = cudaEventRecord(ev, st);
  if (e == cudaSuccess) e = cudaEventSynchronize(ev);
  cudaError_t d = cudaEventDestroy(ev);
  return e != cudaSuccess ? e : d;
}
}  // namespace e2e

namespace {
thread_local e2e::HostTrace* g_trace = nullptr;

bool trace_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("E2E_TRACE");
    return v && v[0] && v[0] != '0';
  }();
  return on;
}

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void usage(double* cpu_ms, long* nv, long* niv) {
  rusage r;
  getrusage(RUSAGE_THREAD, &r);
  *cpu_ms = (r.ru_utime.tv_sec + r.ru_stime.tv_sec) * 1e3 + (r.ru_utime.tv_usec + r.ru_stime.tv_usec) * 1e-3;
  *nv = r.ru_nvcsw;
  *niv = r.ru_nivcsw;
}
}  // namespace

namespace e2e {
HostTrace::HostTrace(const char* nm) : name(nm) {
  if (!trace_enabled()) return;
  on = true;
  cudaMemPool_t pool;
  uint64_t r = 0;
  if (device_pool(&pool) == cudaSuccess && cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r) == cudaSuccess)
    pool0 = r;
  t0 = last = now_ms();
  usage(&cpu0, &nv0, &niv0);
  prev = g_trace;
  g_trace = this;
}

void HostTrace::mark(const char* what) {
  if (!on) return;
  const double t = now_ms();
  char b[96];
  std::snprintf(b, sizeof(b), " %s=%.2f", what, t - last);
  line += b;
  last = t;
}

HostTrace::~HostTrace() {
  if (!on) return;
  g_trace = prev;
  double cpu;
  long nv, niv;
  usage(&cpu, &nv, &niv);
  size_t reserved = 0;
  cudaMemPool_t pool;
  if (device_pool(&pool) == cudaSuccess) {
    uint64_t r = 0;
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r) == cudaSuccess) reserved = r;
  }
  std::fprintf(stderr, "e2e_trace %s wall=%.2f cpu=%.2f vcsw=%ld ivcsw=%ld pool_mb=%.0f->%.0f |%s\n", name,
               now_ms() - t0, cpu - cpu0, nv - nv0, niv - niv0, pool0 / 1048576.0, reserved / 1048576.0,
               line.c_str());
}

void trace_mark(const char* what) {
  if (g_trace) g_trace->mark(what);
}
}  // namespace e2e

extern "C" e2e_status e2e_memory_trim(void) {
  cudaMemPool_t pool;
  cudaError_t e = device_pool(&pool);
  if (e != cudaSuccess) return cuda_fail(e, "device_pool");
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize");
  const int dev = current_device();
  if (dev >= 0) drop_cached(dev, 0);
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceSynchronize");
  e = cudaMemPoolTrimTo(pool, 0);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemPoolTrimTo");
  return E2E_OK;
}

extern "C" int e2e_abi_version(void) { return E2E_DP_ABI_VERSION; }

extern "C" const char* e2e_last_error(void) { return g_err.c_str(); }

extern "C" const char* e2e_status_string(e2e_status st) {
  switch (st) {
    case E2E_OK: return "ok";
    case E2E_ERR_INVALID: return "invalid argument";
    case E2E_ERR_CUDA: return "CUDA error";
    case E2E_ERR_NOMEM: return "out of memory";
    case E2E_ERR_IO: return "I/O error";
    case E2E_ERR_TIMEOUT: return "timeout";
    case E2E_ERR_NOT_CONVERGED: return "not converged";
    case E2E_ERR_UNSUPPORTED: return "unsupported";
    case E2E_ERR_DEVICE: return "device-side check failed";
    case E2E_ERR_CANCELLED: return "cancelled";
    case E2E_ERR_BUSY: return "busy";
  }
  return "unknown status";
}

// ---------------------------------------------------------------------------------
// problem helpers
// ---------------------------------------------------------------------------------
extern "C" e2e_status e2e_problem_from_params(const float pp[32], e2e_problem* o) {
  if (!pp || !o) return fail(E2E_ERR_INVALID, "null argument");
  std::memset(o, 0, sizeof(*o));
  o->gsize = (int32_t)pp[0];
  o->num_actions = (int32_t)pp[1];
  o->nrzns = (int32_t)pp[2];
  o->F = pp[3];
  o->dt = pp[4];
  o->r_outbound = pp[5];
  o->r_terminal = pp[6];
  o->nmodes = (int32_t)pp[7];
  o->i_term = (int32_t)pp[8];
  o->j_term = (int32_t)pp[9];
  o->nt = (int32_t)pp[10];
  o->is_stationary = (int32_t)pp[11];
  o->term_subgrid_size = (int32_t)pp[12];
  o->reward_type = (int32_t)pp[13];
  o->num_ac_speeds = (int32_t)pp[14];
  o->num_ac_angles = (int32_t)pp[15];
  o->dx = pp[16];
  o->dy = pp[17];
  o->neighb_gsize = (int32_t)pp[18];
  o->alpha = pp[19];
  o->x0 = o->dx / 2;  // header convention, src/input_to_build_model.h:14-15
  o->y0 = o->dy / 2;
  return E2E_OK;
}

extern "C" e2e_status e2e_problem_to_params(const e2e_problem* p, float pp[32]) {
  if (!p || !pp) return fail(E2E_ERR_INVALID, "null argument");
  for (int i = 0; i < 32; ++i) pp[i] = -9999.0f;
  pp[0] = (float)p->gsize;
  pp[1] = (float)p->num_actions;
  pp[2] = (float)p->nrzns;
  pp[3] = p->F;
  pp[4] = p->dt;
  pp[5] = p->r_outbound;
  pp[6] = p->r_terminal;
  pp[7] = (float)p->nmodes;
  pp[8] = (float)p->i_term;
  pp[9] = (float)p->j_term;
  pp[10] = (float)p->nt;
  pp[11] = (float)p->is_stationary;
  pp[12] = (float)p->term_subgrid_size;
  pp[13] = (float)p->reward_type;
  pp[14] = (float)p->num_ac_speeds;
  pp[15] = (float)p->num_ac_angles;
  pp[16] = p->dx;
  pp[17] = p->dy;
  pp[18] = (float)p->neighb_gsize;
  pp[19] = p->alpha;
  return E2E_OK;
}

namespace e2e {

e2e_status validate_problem(const e2e_problem* p) {
  if (!p) return fail(E2E_ERR_INVALID, "null problem");
  if (p->gsize < 2 || p->nt < 2) return fail(E2E_ERR_INVALID, "gsize and nt must be >= 2");
  if ((int64_t)p->gsize * p->gsize * p->nt >= ((int64_t)1 << 31))
    return fail(E2E_ERR_UNSUPPORTED, "nt * gsize^2 must be below 2^31 (int32 state indices)");
  if (p->num_ac_speeds < 1 || p->num_ac_angles < 1 ||
      p->num_actions != p->num_ac_speeds * p->num_ac_angles)
    return fail(E2E_ERR_INVALID, "num_actions must equal num_ac_speeds * num_ac_angles");
  if (p->num_actions > 32) return fail(E2E_ERR_UNSUPPORTED, "at most 32 actions are supported");
  if (p->nrzns < 1) return fail(E2E_ERR_INVALID, "nrzns must be >= 1");
  if (p->nrzns > 32767) return fail(E2E_ERR_UNSUPPORTED, "nrzns above 32767 is not supported");
  if (p->nmodes < 0 || p->nmodes > 256) return fail(E2E_ERR_INVALID, "nmodes out of range");
  if (p->neighb_gsize < 1 || p->neighb_gsize % 2 != 1 || p->neighb_gsize > p->gsize)
    return fail(E2E_ERR_INVALID, "neighb_gsize must be odd and <= gsize (src/build_model.cu:1027-1028)");
  if (!(p->dx > 0) || !(p->dy > 0)) return fail(E2E_ERR_INVALID, "dx, dy must be > 0");
  if (p->reward_type < 0 || p->reward_type > 4) return fail(E2E_ERR_INVALID, "reward_type out of range");
  if (p->term_subgrid_size < 0) return fail(E2E_ERR_INVALID, "term_subgrid_size < 0");
  return E2E_OK;
}

void host_ticks(const e2e_problem* p, std::vector<float>& xs, std::vector<float>& ys) {
  // define_xs_or_ys, src/build_model.cu:1395-1399 (float arithmetic)
  xs.resize(p->gsize);
  ys.resize(p->gsize);
  for (int i = 0; i < p->gsize; i++) {
    float fi = (float)i;
    xs[i] = p->x0 + fi * p->dx;
    ys[i] = p->y0 + fi * p->dy;
  }
}

void host_actions(const e2e_problem* p, std::vector<float>& speed, std::vector<float>& angle) {
  // populate_actions / populate_ac_angles / populate_ac_speeds, src/build_model.cu:1403-1457
  const int na = p->num_ac_angles, ns = p->num_ac_speeds;
  std::vector<float> ang(na), spd(ns);
  for (int i = 0; i < na; i++) ang[i] = (float)(i * (2 * M_PI) / na);
  if (ns == 1) {
    spd[0] = p->F;
  } else {
    float delF = p->F / (float)ns;
    for (int i = 0; i < ns; i++) spd[i] = (float)(i + 1) * delF;
  }
  speed.resize(na * ns);
  angle.resize(na * ns);
  for (int i = 0; i < ns; i++)
    for (int j = 0; j < na; j++) {
      int idx = j + na * i;
      speed[idx] = spd[i];
      angle[idx] = ang[j];
    }
}

e2e_status upload(const void* src, size_t bytes, int where, void** dst, bool* owned,
                  cudaStream_t st) {
  if (where == E2E_DEVICE) {
    *dst = const_cast<void*>(src);
    *owned = false;
    return E2E_OK;
  }
  void* d = nullptr;
  CK(dalloc((void**)&d, bytes ? bytes : 16, st));
  if (bytes) {
    cudaError_t e = cudaMemcpyAsync(d, src, bytes, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) {
      dfree(d, st);
      return cuda_fail(e, "cudaMemcpyAsync(fields)");
    }
  }
  *dst = d;
  *owned = true;
  return E2E_OK;
}

// Device copies of xs/ys/actions, shared by build paths.
e2e_status make_dev_problem(const e2e_problem* p, cudaStream_t st, DevProblem* D,
                            DeviceScratch* keep) {
  std::vector<float> xs, ys, speed, angle;
  host_ticks(p, xs, ys);
  host_actions(p, speed, angle);
  const int g = p->gsize, na = p->num_actions;
  size_t bytes = sizeof(float) * (2 * (size_t)g + 4 * (size_t)na);
  float* d = nullptr;
  CK(dalloc((void**)&d, bytes, st));
  keep->add(d);
  std::vector<float> h(2 * (size_t)g + 4 * (size_t)na);
  std::copy(xs.begin(), xs.end(), h.begin());
  std::copy(ys.begin(), ys.end(), h.begin() + g);
  std::copy(speed.begin(), speed.end(), h.begin() + 2 * g);
  std::copy(angle.begin(), angle.end(), h.begin() + 2 * g + na);
  CK(cudaMemcpyAsync(d, h.data(), bytes, cudaMemcpyHostToDevice, st));
  float* dang = d + 2 * g + na;
  float* dcos = d + 2 * g + 2 * na;
  float* dsin = d + 2 * g + 3 * na;
  CK(launch_action_trig(dang, na, dcos, dsin, st));
  std::memset(D, 0, sizeof(*D));
  D->g = g;
  D->nt = p->nt;
  D->nm = p->nmodes;
  D->nrzns = p->nrzns;
  D->na = na;
  D->m = p->neighb_gsize;
  D->del = (p->neighb_gsize - 1) / 2;
  D->it = p->i_term;
  D->jt = p->j_term;
  D->tsg = p->term_subgrid_size;
  D->reward_type = p->reward_type;
  D->dt = p->dt;
  D->r_out = p->r_outbound;
  D->r_term = p->r_terminal;
  D->alpha = p->alpha;
  D->xs0 = xs[0];
  D->xsn = xs[g - 1];
  D->ys0 = ys[0];
  D->ysn = ys[g - 1];
  D->Dj = std::fabs(xs[1] - xs[0]);
  D->Di = std::fabs(ys[1] - ys[0]);
  D->unit_step = (D->Dj == 1.0f && D->Di == 1.0f) ? 1 : 0;
  D->axmax = xs[g - 1] - xs[0];
  D->aymax = -(ys[0] - ys[g - 1]);
  D->xs = d;
  D->ys = d + g;
  D->ac_speed = d + 2 * g;
  D->ac_cos = dcos;
  D->ac_sin = dsin;
  return E2E_OK;
}

int64_t model_bytes(const e2e_model* m) {
  int64_t pb = m->index_bits == 32 ? 4 : 8;
  int64_t cb = m->count_type == E2E_COUNT_U16 ? 2 : 4;
  return (m->n_rows + 1) * pb + m->nnz * (4 + cb) + m->ns * m->na * 4;
}

ViModel vi_model(const e2e_model* m) {
  ViModel M;
  M.ns = m->ns;
  M.n_row_states = m->n_row_states;
  M.na = m->na;
  M.nrzns = m->nrzns;
  M.count_type = m->count_type == E2E_COUNT_U16 ? CNT_U16 : (m->count_type == E2E_COUNT_U32 ? CNT_U32 : VAL_F32);
  M.index_bits = m->index_bits;
  M.row_ptr = m->row_ptr;
  M.col = m->col;
  M.cnt = m->cnt;
  M.R = m->R;
  return M;
}

void free_model_buffers(e2e_model* m) {
  // pool memory, released in stream order on the legacy default stream
  if (m->pack) {
    free_pack(m->pack);
    delete m->pack;
    m->pack = nullptr;
  }
  dfree(m->row_ptr, 0);
  dfree(m->col, 0);
  dfree(m->cnt, 0);
  dfree(m->R, 0);
  dfree(m->sumR, 0);
  m->sumR = nullptr;
  m->row_ptr = nullptr;
  m->col = nullptr;
  m->cnt = nullptr;
  m->R = nullptr;
}

}  // namespace e2e

// ---------------------------------------------------------------------------------
// action table
// ---------------------------------------------------------------------------------
extern "C" e2e_status e2e_action_table(const e2e_problem* p, float* speed, float* angle,
                                       float* cosv, float* sinv) {
  if (!p || p->num_actions < 1 || p->num_actions != p->num_ac_speeds * p->num_ac_angles)
    return fail(E2E_ERR_INVALID, "bad action definition");
  std::vector<float> sp, an;
  host_actions(p, sp, an);
  const int na = p->num_actions;
  if (speed) std::copy(sp.begin(), sp.end(), speed);
  if (angle) std::copy(an.begin(), an.end(), angle);
  if (cosv || sinv) {
    float* d = nullptr;
    CK(cudaMalloc((void**)&d, sizeof(float) * 3 * na));
    cudaError_t e = cudaMemcpy(d, an.data(), sizeof(float) * na, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = launch_action_trig(d, na, d + na, d + 2 * na, 0);
    std::vector<float> h(2 * na);
    if (e == cudaSuccess) e = cudaMemcpy(h.data(), d + na, sizeof(float) * 2 * na, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "e2e_action_table");
    if (cosv) std::copy(h.begin(), h.begin() + na, cosv);
    if (sinv) std::copy(h.begin() + na, h.end(), sinv);
  }
  return E2E_OK;
}

// ---------------------------------------------------------------------------------
// build
// ---------------------------------------------------------------------------------
extern "C" e2e_status e2e_build_model(const e2e_problem* p, const e2e_fields* f, int where,
                                      const e2e_build_opts* opts, e2e_model** out,
                                      void* stream) {
  if (!out) return fail(E2E_ERR_INVALID, "null output handle");
  *out = nullptr;
  e2e_status vs = validate_problem(p);
  if (vs != E2E_OK) return vs;
  if (!f || !f->u || !f->v || !f->yi || !f->s || !f->mask || (p->nmodes > 0 && (!f->ui || !f->vi)))
    return fail(E2E_ERR_INVALID, "null field pointer");
  if (where != E2E_HOST && where != E2E_DEVICE) return fail(E2E_ERR_INVALID, "bad fields_where");
  e2e_build_opts o{};
  o.count_type = E2E_COUNT_AUTO;
  if (opts) o = *opts;
  int count_bits = 16;
  if (o.count_type == E2E_COUNT_U32) count_bits = 32;
  else if (o.count_type == E2E_COUNT_U16 || o.count_type == E2E_COUNT_AUTO) count_bits = 16;
  else return fail(E2E_ERR_INVALID, "count_type must be AUTO, U16 or U32");
  cudaStream_t st = (cudaStream_t)stream;

  BuildPlan plan;
  e2e_status s = plan_build(p, count_bits, o.stage_hint, &plan);
  if (s != E2E_OK) return s;
  plan.keep_sums = o.keep_reward_parts != 0;

  HostTrace trace("build_model");
  DeviceScratch scratch(st);
  FieldsOnDevice fd;
  s = fields_to_device(p, f, where, st, &fd, &scratch, /*defer=*/true);
  if (s != E2E_OK) return s;
  trace.mark("fields");

  e2e_model* m = new (std::nothrow) e2e_model();
  if (!m) return fail(E2E_ERR_NOMEM, "host allocation");
  s = run_build(p, fd, plan, st, &scratch, m);
  if (s != E2E_OK) {
    free_model_buffers(m);
    delete m;
    return s;
  }
  CK(cudaStreamSynchronize(st));
  trace.mark("done");
  *out = m;
  return E2E_OK;
}

namespace e2e {

e2e_status plan_build(const e2e_problem* p, int count_bits, int64_t stage_hint, BuildPlan* pl) {
  pl->count_bits = count_bits;
  pl->ncells = (int64_t)p->gsize * p->gsize;
  pl->ns = pl->ncells * p->nt;
  pl->na = p->num_actions;
  pl->n_rows = (int64_t)(p->nt - 1) * pl->ncells * pl->na;
  pl->tiles_per_layer = (pl->ncells + 31) / 32;  // builder CTAs per layer
  {
    const int nwarps = 1 << build_lanes_log2(pl->na);  // emission tiles (warps) per CTA
    pl->cells_per_tile = 32 / nwarps;
    pl->etiles_per_layer = pl->tiles_per_layer * nwarps;
    pl->n_tiles = pl->etiles_per_layer * (p->nt - 1);
  }
  // realisations per velocity chunk: 128 for unit spacing (no mask table)
  // while two 512-thread CTAs still fit an SM, else 64; halved while the
  // need exceeds 200 KB
  bool unit;
  {  // the test of make_dev_problem (unit_step) on the same ticks
    std::vector<float> xs, ys;
    host_ticks(p, xs, ys);
    unit = std::fabs(xs[1] - xs[0]) == 1.0f && std::fabs(ys[1] - ys[0]) == 1.0f;
  }
  pl->rc = unit ? 128 : 64;
  size_t sm = build_smem_bytes(pl->na, p->nmodes, pl->rc, unit, 1);
  if (unit && pl->na <= 16 && sm > 112 * 1024) {
    pl->rc = 64;
    sm = build_smem_bytes(pl->na, p->nmodes, pl->rc, unit, 1);
  }
  while (sm > 200 * 1024 && pl->rc > 16) {
    pl->rc /= 2;
    sm = build_smem_bytes(pl->na, p->nmodes, pl->rc, unit, 1);
  }
  if (sm > 220 * 1024) return fail(E2E_ERR_UNSUPPORTED, "shared memory need too large (nmodes/actions)");
  // A second coefficient buffer lets the chunk loop stage chunk c+1 while
  // chunk c is read, with one CTA barrier a chunk instead of two; taken only
  // when it costs no builder CTA per SM.
  pl->ybufs = 1;
  {
    const size_t sm2 = build_smem_bytes(pl->na, p->nmodes, pl->rc, unit, 2);
    if (sm2 <= 220 * 1024) {
      const int c1 = build_ctas_per_sm(pl->na, sm, unit);
      if (c1 > 0 && build_ctas_per_sm(pl->na, sm2, unit) >= c1) pl->ybufs = 2;
    }
  }
  if (pl->tiles_per_layer > 0x7fffffff || p->nt - 1 > 65535)
    return fail(E2E_ERR_UNSUPPORTED, "grid too large for one launch");
  pl->stage_cap = stage_hint > 0 ? stage_hint : pl->n_rows * 4 + 4096;
  pl->pool_units = std::min<int64_t>(std::max<int64_t>(pl->n_rows / 64, 256), 8192);
  return E2E_OK;
}

e2e_status fields_to_device(const e2e_problem* p, const e2e_fields* f, int where,
                            cudaStream_t st, FieldsOnDevice* fd, DeviceScratch* keep, bool defer) {
  const size_t nc = (size_t)p->gsize * p->gsize, nt = (size_t)p->nt, nm = (size_t)p->nmodes;
  const size_t b2 = sizeof(float) * nt * nc;
  const size_t bm = sizeof(float) * nt * nm * nc;
  const size_t by = sizeof(float) * nt * (size_t)p->nrzns * nm;
  const void* src[7] = {f->u, f->v, f->ui, f->vi, f->yi, f->s, f->mask};
  const size_t bytes[7] = {b2, b2, bm, bm, by, b2, sizeof(int32_t) * nt * nc};
  void* dst[7];
  const bool deferred = defer && where == E2E_HOST;
  fd->nt = (int)nt;
  for (int k = 0; k < 7; ++k) {
    bool owned = false;
    if (!src[k]) {
      dst[k] = nullptr;
      continue;
    }
    if (deferred) {  // allocate now, copy per range of time steps later
      CK(dalloc(&dst[k], bytes[k] ? bytes[k] : 16, st));
      keep->add(dst[k]);
      fd->src[k] = src[k];
      fd->dst[k] = dst[k];
      fd->step_bytes[k] = bytes[k] / nt;
      fd->n_deferred++;
      fd->h2d_bytes += bytes[k];
      continue;
    }
    e2e_status s = upload(src[k], bytes[k], where, &dst[k], &owned, st);
    if (s != E2E_OK) return s;
    if (owned) keep->add(dst[k]);
    fd->h2d_bytes += owned ? bytes[k] : 0;
  }
  fd->F.u = (const float*)dst[0];
  fd->F.v = (const float*)dst[1];
  fd->F.ui = (const float*)dst[2];
  fd->F.vi = (const float*)dst[3];
  fd->F.Y = (const float*)dst[4];
  fd->F.s = (const float*)dst[5];
  fd->F.mask = (const int32_t*)dst[6];
  return E2E_OK;
}

e2e_status copy_field_steps(const FieldsOnDevice& fd, int t0, int t1, cudaStream_t st) {
  if (t1 <= t0) return E2E_OK;
  for (int k = 0; k < 7; ++k) {
    if (!fd.src[k]) continue;
    const size_t off = fd.step_bytes[k] * (size_t)t0, n = fd.step_bytes[k] * (size_t)(t1 - t0);
    CK(cudaMemcpyAsync(static_cast<char*>(fd.dst[k]) + off, static_cast<const char*>(fd.src[k]) + off, n,
                       cudaMemcpyHostToDevice, st));
  }
  return E2E_OK;
}

e2e_status run_build(const e2e_problem* p, const FieldsOnDevice& fd, const BuildPlan& pl,
                     cudaStream_t st, DeviceScratch* scratch, e2e_model* m) {
  const DevFields& F = fd.F;
  DevProblem D;
  e2e_status s = make_dev_problem(p, st, &D, scratch);
  if (s != E2E_OK) return s;
  const int cbytes = pl.count_bits == 16 ? 2 : 4;
  // model R (state-major, last layer zero as src/build_model.cu:1173-1176)
  CK(dalloc((void**)&m->R, sizeof(float) * (size_t)pl.ns * pl.na, st));
  CK(cudaMemsetAsync(m->R, 0, sizeof(float) * (size_t)pl.ns * pl.na, st));
  if (pl.keep_sums) {
    CK(dalloc((void**)&m->sumR, sizeof(float) * (size_t)pl.ns * pl.na, st));
    CK(cudaMemsetAsync(m->sumR, 0, sizeof(float) * (size_t)pl.ns * pl.na, st));
  }
  uint32_t* row_off = nullptr;
  int64_t* tile_base = nullptr;
  int32_t* tile_len = nullptr;
  unsigned long long* ctr = nullptr;
  CK(dalloc((void**)&row_off, sizeof(uint32_t) * (size_t)std::max<int64_t>(pl.n_rows, 1), st));
  scratch->add(row_off);
  CK(dalloc((void**)&tile_base, sizeof(int64_t) * (size_t)std::max<int64_t>(pl.n_tiles, 1), st));
  scratch->add(tile_base);
  CK(dalloc((void**)&tile_len, sizeof(int32_t) * (size_t)std::max<int64_t>(pl.n_tiles, 1), st));
  scratch->add(tile_len);
  CK(dalloc((void**)&ctr, sizeof(unsigned long long) * CTR_COUNT, st));
  scratch->add(ctr);

  int64_t cap = pl.stage_cap, pool_units = pl.pool_units;
  int32_t* stage_col = nullptr;
  void* stage_cnt = nullptr;
  uint32_t* pool = nullptr;
  unsigned long long hc[CTR_COUNT];
  const int mm = p->neighb_gsize * p->neighb_gsize;
  cudaEvent_t ev[4];
  for (int k = 0; k < 4; ++k) CK(cudaEventCreate(&ev[k]));
  trace_mark("events");
  struct EvFree {
    cudaEvent_t* e;
    ~EvFree() { for (int k = 0; k < 4; ++k) cudaEventDestroy(e[k]); }
  } evfree{ev};
  trace_mark("setup");
  for (int attempt = 0; attempt < 3; ++attempt) {
    if (!stage_col) {
      CK(dalloc((void**)&stage_col, sizeof(int32_t) * (size_t)cap, st));
      CK(dalloc((void**)&stage_cnt, (size_t)cbytes * (size_t)cap, st));
    }
    if (!pool) CK(dalloc((void**)&pool, sizeof(uint32_t) * (size_t)mm * (size_t)pool_units, st));
    CK(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long) * CTR_COUNT, st));
    BuildArgs A;
    A.P = D;
    A.F = F;
    A.t0 = 0;
    A.tiles_per_layer = (int)pl.tiles_per_layer;
    A.rc = pl.rc;
    A.ybufs = pl.ybufs;
    A.lanes_log2 = build_lanes_log2(pl.na);
    A.stage_col = stage_col;
    A.stage_cnt = stage_cnt;
    A.stage_cap = cap;
    A.counters = ctr;
    A.row_off = row_off;
    A.tile_base = tile_base;
    A.tile_len = tile_len;
    A.R = m->R;
    A.sumR = m->sumR;
    A.pool = pool;
    A.pool_units = pool_units;
    CK(cudaEventRecord(ev[0], st));
    trace_mark("buffers");
    if (attempt == 0 && fd.n_deferred) {
      // host fields: copy the first layers' steps, then build them while the
      // rest is copied on a second stream, then build the remaining layers
      const int la = std::max(1, std::min(p->nt - 1, (p->nt - 1) / 16));
      e2e_status cs = copy_field_steps(fd, 0, la + 1, st);
      if (cs != E2E_OK) return cs;
      cudaStream_t cps = nullptr;
      cudaEvent_t evs[2] = {nullptr, nullptr};
      struct CopyFree {
        cudaStream_t* s;
        cudaEvent_t* e;
        ~CopyFree() {
          for (int k = 0; k < 2; ++k)
            if (e[k]) cudaEventDestroy(e[k]);
          if (*s) cudaStreamDestroy(*s);
        }
      } cpfree{&cps, evs};
      if (la < p->nt - 1) {
        CK(cudaStreamCreateWithFlags(&cps, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k) CK(cudaEventCreateWithFlags(&evs[k], cudaEventDisableTiming));
        // after the buffers exist (stream-ordered allocations) and the first
        // steps are in, before the first launch, so the copy runs beside it
        CK(cudaEventRecord(evs[0], st));
        CK(cudaStreamWaitEvent(cps, evs[0], 0));
        trace_mark("copy_stream");
        cs = copy_field_steps(fd, la + 1, p->nt, cps);
        if (cs != E2E_OK) return cs;
        CK(cudaEventRecord(evs[1], cps));
        trace_mark("copies");
      }
      BuildArgs A0 = A;
      CK(launch_build_tiles(A0, pl.count_bits, la, st));
      m->build_launches++;
      trace_mark("first_layers");
      if (la < p->nt - 1) {
        CK(cudaStreamWaitEvent(st, evs[1], 0));
        BuildArgs A1 = A;
        A1.t0 = la;
        CK(launch_build_tiles(A1, pl.count_bits, p->nt - 1 - la, st));
        m->build_launches++;
      }
    } else {
      CK(launch_build_tiles(A, pl.count_bits, p->nt - 1, st));
      m->build_launches++;
    }
    trace_mark("launch");
    CK(cudaEventRecord(ev[1], st));
    trace_mark("record");
    // sleep through the builder; the counters' copy into host (stack) memory
    // would otherwise spin until it finishes
    CK(sleep_sync(st));
    trace_mark("build");
    CK(cudaMemcpyAsync(hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    trace_mark("counters");
    bool again = false;
    if (hc[CTR_FLAGS] & FLAG_POOL_EXHAUSTED) {
      dfree(pool, st);
      pool = nullptr;
      pool_units = (int64_t)hc[CTR_POOL];
      if ((double)pool_units * mm * 4 > 32.0 * (1ull << 30))
        return fail(E2E_ERR_UNSUPPORTED, "transition spread too wide: dense-histogram pool above 32 GiB");
      again = true;
    }
    if ((int64_t)hc[CTR_STAGE] > cap) {
      dfree(stage_col, st);
      dfree(stage_cnt, st);
      stage_col = nullptr;
      stage_cnt = nullptr;
      cap = (int64_t)hc[CTR_STAGE];
      again = true;
    }
    if (!again) break;
    if (attempt == 2) return fail(E2E_ERR_DEVICE, "builder did not settle after re-runs");
  }
  scratch->add(stage_col);
  scratch->add(stage_cnt);
  scratch->add(pool);
  const int64_t nnz = (int64_t)hc[CTR_STAGE];
  m->ns = pl.ns;
  m->n_rows = pl.n_rows;
  m->n_row_states = pl.ns - pl.ncells;
  m->nnz = nnz;
  m->na = pl.na;
  m->nt = p->nt;
  m->ncells = (int32_t)pl.ncells;
  m->nrzns = p->nrzns;
  m->count_type = pl.count_bits == 16 ? E2E_COUNT_U16 : E2E_COUNT_U32;
  m->index_bits = nnz < ((int64_t)1 << 31) ? 32 : 64;
  m->dropped = hc[CTR_DROPPED];
  m->misbinned = hc[CTR_MISBIN];
  m->overflow_rows = hc[CTR_OVERFLOW_ROWS];
  m->layered = true;
  m->prob = *p;
  m->has_prob = true;
  const int pb = m->index_bits == 32 ? 4 : 8;
  CK(dalloc(&m->row_ptr, (size_t)pb * (size_t)(pl.n_rows + 1), st));
  CK(dalloc((void**)&m->col, sizeof(int32_t) * (size_t)(nnz + 16), st));
  CK(dalloc(&m->cnt, (size_t)cbytes * (size_t)(nnz + 16), st));
  trace_mark("model_alloc");
  int64_t* canon = nullptr;
  int64_t* total = nullptr;
  CK(dalloc((void**)&canon, sizeof(int64_t) * (size_t)std::max<int64_t>(pl.n_tiles, 1), st));
  scratch->add(canon);
  CK(dalloc((void**)&total, sizeof(int64_t), st));
  scratch->add(total);
  CK(cudaEventRecord(ev[2], st));
  int64_t* block_sums = nullptr;
  CK(dalloc((void**)&block_sums, sizeof(int64_t) * (size_t)(pl.n_tiles / 1024 + 2), st));
  scratch->add(block_sums);
  trace_mark("scratch_alloc");
  CK(launch_scan_tiles(tile_len, pl.n_tiles, canon, total, block_sums, st));
  trace_mark("scan_launch");
  AssembleArgs S;
  S.n_tiles = pl.n_tiles;
  S.tiles_per_layer = pl.etiles_per_layer;
  S.cells_per_tile = pl.cells_per_tile;
  S.ncells = pl.ncells;
  S.n_rows = pl.n_rows;
  S.total_nnz = nnz;
  S.na = pl.na;
  S.tile_base = tile_base;
  S.tile_len = tile_len;
  S.canon = canon;
  S.row_off = row_off;
  S.stage_col = stage_col;
  S.stage_cnt = stage_cnt;
  S.row_ptr = m->row_ptr;
  S.col = m->col;
  S.cnt = m->cnt;
  CK(launch_assemble(S, pl.count_bits, m->index_bits, st));
  CK(cudaEventRecord(ev[3], st));
  trace_mark("assemble_launch");
  CK(cudaEventSynchronize(ev[3]));
  trace_mark("assemble");
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
  m->build_kernel_ms = ms;
  CK(cudaEventElapsedTime(&ms, ev[2], ev[3]));
  m->assemble_ms = ms;
  return E2E_OK;
}

}  // namespace e2e

extern "C" e2e_status e2e_model_free(e2e_model* m) {
  if (!m) return E2E_OK;
  free_model_buffers(m);
  delete m;
  return E2E_OK;
}

extern "C" e2e_status e2e_model_get_info(const e2e_model* m, e2e_model_info* info) {
  if (!m || !info) return fail(E2E_ERR_INVALID, "null argument");
  std::memset(info, 0, sizeof(*info));
  info->ns = m->ns;
  info->n_rows = m->n_rows;
  info->nnz = m->nnz;
  info->num_actions = m->na;
  info->nt = m->nt;
  info->ncells = m->ncells;
  info->nrzns = m->nrzns;
  info->count_type = m->count_type;
  info->index_bits = m->index_bits;
  info->row_ptr = m->row_ptr;
  info->col = m->col;
  info->cnt = m->cnt;
  info->R = m->R;
  info->dropped = m->dropped;
  info->overflow_units = m->overflow_rows;
  info->build_kernel_ms = m->build_kernel_ms;
  info->assemble_ms = m->assemble_ms;
  info->build_launches = m->build_launches;
  return E2E_OK;
}

extern "C" e2e_status e2e_model_copy_to_host(const e2e_model* m, int64_t* row_ptr, int32_t* col,
                                             uint32_t* cnt, float* R, void* stream) {
  if (!m) return fail(E2E_ERR_INVALID, "null model");
  cudaStream_t st = (cudaStream_t)stream;
  if (row_ptr) {
    if (m->index_bits == 64) {
      CK(cudaMemcpyAsync(row_ptr, m->row_ptr, sizeof(int64_t) * (m->n_rows + 1), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
    } else {
      std::vector<int32_t> t((size_t)m->n_rows + 1);
      CK(cudaMemcpyAsync(t.data(), m->row_ptr, sizeof(int32_t) * t.size(), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      for (size_t i = 0; i < t.size(); ++i) row_ptr[i] = t[i];
    }
  }
  if (col && m->nnz)
    CK(cudaMemcpyAsync(col, m->col, sizeof(int32_t) * m->nnz, cudaMemcpyDeviceToHost, st));
  if (cnt && m->nnz) {
    if (m->count_type == E2E_COUNT_U16) {
      std::vector<uint16_t> t((size_t)m->nnz);
      CK(cudaMemcpyAsync(t.data(), m->cnt, sizeof(uint16_t) * t.size(), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      for (size_t i = 0; i < t.size(); ++i) cnt[i] = t[i];
    } else {
      CK(cudaMemcpyAsync(cnt, m->cnt, sizeof(uint32_t) * m->nnz, cudaMemcpyDeviceToHost, st));
    }
  }
  if (R) CK(cudaMemcpyAsync(R, m->R, sizeof(float) * m->ns * m->na, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return E2E_OK;
}

// ---------------------------------------------------------------------------------
// solve
// ---------------------------------------------------------------------------------
namespace e2e {

// The sliced copy of the model that the sweeps stream (built once per model).
e2e_status ensure_pack(const e2e_model* m, double* pack_ms, cudaStream_t st) {
  *pack_ms = 0.0;
  if (m->pack) return E2E_OK;
  const ViModel M = vi_model(m);
  const bool geo = m->layered && m->has_prob && m->ncells > 0 &&
                   (int64_t)m->prob.gsize * m->prob.gsize == m->ncells;
  const int g = geo ? m->prob.gsize : 0;
  const int del = geo ? (m->prob.neighb_gsize - 1) / 2 : 0;
  const int64_t nc = m->layered ? m->ncells : 0;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  struct EvGuard {
    cudaEvent_t a, b;
    ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
  } evg{e0, e1};
  auto* ps = new PackStore();
  CK(cudaEventRecord(e0, st));
  cudaError_t e = build_pack(M, nc, g, del, ps, st);
  if (e != cudaSuccess) {
    free_pack(ps);
    delete ps;
    return cuda_fail(e, "build_pack");
  }
  CK(cudaEventRecord(e1, st));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  *pack_ms = ms;
  m->pack = ps;
  return E2E_OK;
}

e2e_status solve_on_device(const e2e_model* m, const e2e_vi_opts& o, float* dV, int32_t* dpi,
                           e2e_vi_stats* stats, cudaStream_t st) {
  const int64_t ns = m->ns;
  const int gsel = o.schedule & 15;
  if ((o.schedule & ~0x1ff) || (gsel != 0 && gsel != 1 && gsel != 2 && gsel != 4 && gsel != 8))
    return fail(E2E_ERR_INVALID,
                "schedule: bits 0-3 warps per chunk (0, 1, 2, 4, 8), bits 4-7 sweep tuning, bit 8 tuning given");
  // sweep tuning: given, or the defaults measured on B200 (layered: look-ahead
  // kernel, next layer's chunks prefetched into L2; Jacobi: lean kernel)
  const bool tune_given = (o.schedule & 0x100) != 0;
  const int tune_layered = tune_given ? (o.schedule >> 4) & 15 : VI_TUNE_PF_NEXT;
  const int tune_jacobi = tune_given ? (o.schedule >> 4) & 15 : VI_TUNE_LEAN;
  double pack_ms = 0.0;
  {
    e2e_status ps = ensure_pack(m, &pack_ms, st);
    if (ps != E2E_OK) return ps;
  }
  trace_mark("pack");
  const ViPack& P = m->pack->v;
  DeviceScratch scratch(st);
  float* W = nullptr;
  unsigned long long* resid = nullptr;
  const int max_iter = o.max_iter > 0 ? o.max_iter : (m->nt > 0 ? m->nt + 2 : 100000);
  CK(dalloc((void**)&W, sizeof(float) * (size_t)ns, st));
  scratch.add(W);
  CK(dalloc((void**)&resid, sizeof(unsigned long long) * (size_t)(max_iter + 3), st));
  scratch.add(resid);
  CK(cudaMemsetAsync(resid, 0, sizeof(unsigned long long) * (size_t)(max_iter + 3), st));
  // last slot: barrier count and error bits of the persistent layered sweep
  unsigned int* syncw = reinterpret_cast<unsigned int*>(resid + max_iter + 2);
  cudaEvent_t e0, e1, e2;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventCreate(&e2));
  struct EvGuard {
    cudaEvent_t a, b, c;
    ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); cudaEventDestroy(c); }
  } evg{e0, e1, e2};
  auto t_start = std::chrono::steady_clock::now();
  int iters = 0;
  double last_res = 0.0;
  bool layered_pass = false;
  const int64_t pbytes = m->index_bits == 32 ? 4 : 8;
  const int64_t cbytes = m->count_type == E2E_COUNT_U16 ? 2 : 4;
  int64_t sweep_bytes = (m->n_rows + 1) * pbytes + m->nnz * (4 + cbytes) + ns * m->na * 4 + ns * 12;
  CK(cudaEventRecord(e0, st));
  if (o.method == 1) {
    if (!m->layered || m->ncells <= 0 || m->nt <= 0 || P.nlayers < 2)
      return fail(E2E_ERR_UNSUPPORTED, "layered solve needs a time-layered model (nt, ncells known)");
    // all layers, last first, in one cooperative launch
    CK(launch_vi_layered(P, dV, dpi, syncw, gsel, st, tune_layered));
    CK(cudaEventRecord(e2, st));
    layered_pass = true;
    // verification sweep (Jacobi from the fixed point): residual must be 0
    int32_t* pi2 = nullptr;
    CK(dalloc((void**)&pi2, sizeof(int32_t) * (size_t)ns, st));
    scratch.add(pi2);
    CK(launch_vi_chunks(P, 0, P.nchunks, dV, W, pi2, resid, st, tune_jacobi, syncw + 1));
    unsigned long long h = 0;
    CK(cudaMemcpyAsync(&h, resid, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaEventRecord(e1, st));
    CK(cudaStreamSynchronize(st));
    std::memcpy(&last_res, &h, sizeof(double));
    iters = 2;
  } else {
    float* a = dV;
    float* b = W;
    CK(cudaMemsetAsync(a, 0, sizeof(float) * (size_t)ns, st));
    bool done = false;
    while (!done) {
      if (iters >= max_iter) break;
      ++iters;
      CK(launch_vi_chunks(P, 0, P.nchunks, a, b, dpi, resid + iters, st, tune_jacobi, syncw + 1));
      unsigned long long h = 0;
      CK(cudaMemcpyAsync(&h, resid + iters, sizeof(h), cudaMemcpyDeviceToHost, st));
      CK(cudaStreamSynchronize(st));
      std::memcpy(&last_res, &h, sizeof(double));
      std::swap(a, b);
      if (last_res < (double)o.threshold) done = true;
      if (o.timeout_s > 0) {
        double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
        if (!done && el > o.timeout_s) {
          if (a != dV) CK(cudaMemcpyAsync(dV, a, sizeof(float) * ns, cudaMemcpyDeviceToDevice, st));
          CK(cudaStreamSynchronize(st));
          if (stats) stats->iterations = iters;
          return fail(E2E_ERR_TIMEOUT, "value iteration exceeded timeout_s");
        }
      }
    }
    if (a != dV) CK(cudaMemcpyAsync(dV, a, sizeof(float) * (size_t)ns, cudaMemcpyDeviceToDevice, st));
    CK(cudaEventRecord(e1, st));
    CK(cudaStreamSynchronize(st));
    if (!done) {
      if (stats) {
        stats->iterations = iters;
        stats->residual = last_res;
      }
      return fail(E2E_ERR_NOT_CONVERGED, "max_iter reached before the threshold");
    }
  }
  {
    unsigned int herr = 0;
    CK(cudaMemcpyAsync(&herr, syncw + 1, sizeof(herr), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr) return fail(E2E_ERR_DEVICE, "a bounded device-side wait of the sweep gave up");
  }
  float ms = 0.f, ms_pass = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  if (layered_pass) CK(cudaEventElapsedTime(&ms_pass, e0, e2));
  if (stats) {
    stats->iterations = iters;
    stats->residual = last_res;
    stats->seconds = ms * 1e-3;
    stats->bytes_per_sweep = sweep_bytes;
    stats->stream_bytes_per_sweep = pack_sweep_bytes(P);
    stats->pack_ms = pack_ms;
    stats->sweep_seconds = ms_pass * 1e-3;
    stats->fp64_max_abs_err = 0;
    stats->fp64_max_rel_err = 0;
  }
  if (o.fp64_check) {
    if (!m->layered) return fail(E2E_ERR_UNSUPPORTED, "fp64 check needs a time-layered model");
    const ViModel M = vi_model(m);
    double* Vd = nullptr;
    unsigned long long* err = nullptr;
    CK(dalloc((void**)&Vd, sizeof(double) * (size_t)ns, st));
    scratch.add(Vd);
    CK(dalloc((void**)&err, sizeof(unsigned long long) * 2, st));
    scratch.add(err);
    CK(cudaMemsetAsync(err, 0, sizeof(unsigned long long) * 2, st));
    const int64_t nc = m->ncells;
    CK(launch_vi_sweep_f64(M, m->n_row_states, ns, Vd, st));
    for (int64_t t = (m->n_row_states / nc) - 1; t >= 0; --t)
      CK(launch_vi_sweep_f64(M, t * nc, (t + 1) * nc, Vd, st));
    CK(launch_compare_f64(dV, Vd, ns, err, st));
    unsigned long long h[2];
    CK(cudaMemcpyAsync(h, err, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double ea, er;
    std::memcpy(&ea, &h[0], 8);
    std::memcpy(&er, &h[1], 8);
    if (stats) {
      stats->fp64_max_abs_err = ea;
      stats->fp64_max_rel_err = er > 0 ? ea / er : ea;
    }
  }
  return E2E_OK;
}

}  // namespace e2e

extern "C" e2e_status e2e_spvi_solve(const e2e_model* m, const e2e_vi_opts* opts,
                                     int32_t* policy_out, float* value_out, int out_where,
                                     e2e_vi_stats* stats, void* stream) {
  if (!m) return fail(E2E_ERR_INVALID, "null model");
  if (out_where != E2E_HOST && out_where != E2E_DEVICE) return fail(E2E_ERR_INVALID, "bad out_where");
  e2e_vi_opts o{};
  o.method = m->layered ? 1 : 0;
  o.threshold = 0.1f;  // s_stopping_thresh, src/spvi_2.cu:757
  if (opts) o = *opts;
  if (o.method != 0 && o.method != 1) return fail(E2E_ERR_INVALID, "method must be 0 or 1");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t ns = m->ns;
  float* dV = nullptr;
  int32_t* dpi = nullptr;
  HostTrace trace("spvi_solve");
  DeviceScratch scratch(st);
  if (out_where == E2E_DEVICE && value_out) {
    dV = value_out;
  } else {
    CK(dalloc((void**)&dV, sizeof(float) * (size_t)ns, st));
    scratch.add(dV);
  }
  if (out_where == E2E_DEVICE && policy_out) {
    dpi = policy_out;
  } else {
    CK(dalloc((void**)&dpi, sizeof(int32_t) * (size_t)ns, st));
    scratch.add(dpi);
  }
  e2e_status s = solve_on_device(m, o, dV, dpi, stats, st);
  if (s != E2E_OK && s != E2E_ERR_NOT_CONVERGED && s != E2E_ERR_TIMEOUT) return s;
  trace.mark("solve");
  if (out_where == E2E_HOST) {
    if (value_out) CK(cudaMemcpyAsync(value_out, dV, sizeof(float) * ns, cudaMemcpyDeviceToHost, st));
    if (policy_out) CK(cudaMemcpyAsync(policy_out, dpi, sizeof(int32_t) * ns, cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  trace.mark("outputs");
  return s;
}
