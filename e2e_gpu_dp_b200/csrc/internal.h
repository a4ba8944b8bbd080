// Host-side internals shared by the C ABI translation units.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "e2e_dp.h"
#include "kernels.h"

// The model handle behind the opaque e2e_model of the public header.
struct e2e_model {
  int64_t ns = 0;            // states
  int64_t n_rows = 0;        // rows (s, a) stored: n_row_states * na
  int64_t n_row_states = 0;  // states that own rows; later states have Q = R only
  int64_t nnz = 0;
  int32_t na = 0, nt = 0, ncells = 0, nrzns = 1;
  int32_t count_type = E2E_COUNT_U16;
  int32_t index_bits = 32;
  void* row_ptr = nullptr;   // device
  int32_t* col = nullptr;    // device
  void* cnt = nullptr;       // device
  float* R = nullptr;        // device, ns * na (state-major)
  float* sumR = nullptr;     // device, ns * na: reward sums (keep_reward_parts), or null
  uint64_t dropped = 0, misbinned = 0, overflow_rows = 0;
  double build_kernel_ms = 0, assemble_ms = 0;
  int32_t build_launches = 0;
  bool layered = false;      // every transition of a layer-t state leads into layer t+1
  e2e_problem prob{};
  bool has_prob = false;
  // sliced copy for value iteration, built by the first solve that needs it
  mutable e2e::PackStore* pack = nullptr;
};

namespace e2e {

e2e_status fail(e2e_status st, const std::string& msg);
// device allocation from the library's stream-ordered pool, large blocks through
// the library's block cache; release with dfree on the stream that last uses it
cudaError_t dalloc(void** p, size_t bytes, cudaStream_t st);
void dfree(void* p, cudaStream_t st);
e2e_status cuda_fail(cudaError_t e, const char* what);
// wait for the work queued on st with the calling thread asleep (a blocking-sync
// event) rather than spinning: for waits on long builder launches
cudaError_t sleep_sync(cudaStream_t st);

// Host-side phase trace, for finding where a call's wall time goes: with
// E2E_TRACE=1 in the environment, each traced call prints one line to stderr
// with the milliseconds between its marks, its wall and CPU time, its voluntary
// and involuntary context switches, and the bytes the device pool holds.  Off,
// a mark is one branch on a thread-local pointer.
struct HostTrace {
  explicit HostTrace(const char* name);
  ~HostTrace();
  HostTrace(const HostTrace&) = delete;
  HostTrace& operator=(const HostTrace&) = delete;
  void mark(const char* what);
  bool on = false;
  const char* name;
  double t0 = 0, last = 0, cpu0 = 0;
  size_t pool0 = 0;
  long nv0 = 0, niv0 = 0;
  HostTrace* prev = nullptr;
  std::string line;
};
// mark on the trace active on this thread, if any
void trace_mark(const char* what);

// Stream-ordered temporaries released when the owner goes out of scope.
struct DeviceScratch {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit DeviceScratch(cudaStream_t s) : st(s) {}
  void add(void* p) {
    if (p) ptrs.push_back(p);
  }
  ~DeviceScratch() {
    for (void* p : ptrs) dfree(p, st);
  }
  DeviceScratch(const DeviceScratch&) = delete;
  DeviceScratch& operator=(const DeviceScratch&) = delete;
};

struct BuildPlan {
  int count_bits = 16;
  int64_t ncells = 0, ns = 0, n_rows = 0, tiles_per_layer = 0, n_tiles = 0;
  int64_t etiles_per_layer = 0, cells_per_tile = 32;  // emission tiles (one per builder warp)
  int na = 0, rc = 128;
  int ybufs = 1;  // coefficient buffers of the builder's chunk loop (2 when occupancy allows)
  int64_t stage_cap = 0, pool_units = 0;
  bool keep_sums = false;  // keep per-row reward sums (e2e_build_opts.keep_reward_parts)
};

struct FieldsOnDevice {
  DevFields F{};
  size_t h2d_bytes = 0;
  // host fields uploaded later, a range of time steps at a time (fields_to_device
  // with defer): per field the host source, its device buffer and the bytes of
  // one time step (every field is time-major)
  int n_deferred = 0, nt = 0;
  const void* src[7] = {};
  void* dst[7] = {};
  size_t step_bytes[7] = {};
};

e2e_status validate_problem(const e2e_problem* p);
void host_ticks(const e2e_problem* p, std::vector<float>& xs, std::vector<float>& ys);
void host_actions(const e2e_problem* p, std::vector<float>& speed, std::vector<float>& angle);
e2e_status make_dev_problem(const e2e_problem* p, cudaStream_t st, DevProblem* D,
                            DeviceScratch* keep);
e2e_status plan_build(const e2e_problem* p, int count_bits, int64_t stage_hint, BuildPlan* pl);
e2e_status fields_to_device(const e2e_problem* p, const e2e_fields* f, int where, cudaStream_t st,
                            FieldsOnDevice* fd, DeviceScratch* keep, bool defer = false);
// copy time steps [t0, t1) of deferred host fields on stream st
e2e_status copy_field_steps(const FieldsOnDevice& fd, int t0, int t1, cudaStream_t st);
// the build; with deferred host fields the first layers' fields are copied
// first and the rest overlaps the builder's first launch
e2e_status run_build(const e2e_problem* p, const FieldsOnDevice& fd, const BuildPlan& pl,
                     cudaStream_t st, DeviceScratch* scratch, e2e_model* m);
ViModel vi_model(const e2e_model* m);
void free_model_buffers(e2e_model* m);
int64_t model_bytes(const e2e_model* m);
e2e_status solve_on_device(const e2e_model* m, const e2e_vi_opts& o, float* dV, int32_t* dpi,
                           e2e_vi_stats* stats, cudaStream_t st);
// build the model's sliced copy for the sweeps if it has none yet
e2e_status ensure_pack(const e2e_model* m, double* pack_ms, cudaStream_t st);

// One layered solve of a batch: a model, its outputs and, for a served
// request, the re-targeted R around its target (ViJob fields).
struct BatchJobSpec {
  const e2e_model* m = nullptr;
  float* V = nullptr;
  int32_t* pi = nullptr;
  const float* Rwin = nullptr;
  int ti = 0, tj = 0, tsg = 0, wi0 = 0, wj0 = 0, wh = 0, ww = 0;
};
struct BatchResult {
  int launches = 0, groups = 0, tune = 0, grid = 0, graph = 0;
  double seconds = 0, pack_ms = 0, tune_ms = 0;
  int64_t stream_bytes = 0;
};
// schedule: e2e_vi_opts.schedule (bit 9: direct launch instead of a CUDA graph)
e2e_status solve_batch(const std::vector<BatchJobSpec>& jobs, int schedule, cudaStream_t st,
                       BatchResult* res);

}  // namespace e2e
