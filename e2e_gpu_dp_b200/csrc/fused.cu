// Build and solve in one backward pass, never storing the transition model.
//
// The reference builds every (t, a) block of the model (src/build_model.cu:
// 696-892), writes it to disk, and spvi_2 reads it back and iterates
// (src/spvi_2.cu:650-726).  Transitions only go from layer t to t+1
// (src/build_model.cu:635) and the last layer has no rows (:1173-1176), so the
// values of layer t are final as soon as layer t+1's are: the layered schedule
// reaches the Jacobi fixed point in one pass.  Here each layer's rows are built
// by K1 and backed up in its epilogue from the counters still in shared memory
// (launch_build_fused): one cooperative launch whose CTAs take the tiles of
// layers nt-2 down to 0 in order, each tile waiting (bounded) before its
// backup only for the rows of the layer after its own that the backup reads,
// so a layer's sampling overlaps the completion of the next one.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "e2e_dp.h"
#include "internal.h"
#include "kernels.h"

using namespace e2e;

#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

extern "C" e2e_status e2e_build_solve(const e2e_problem* p, const e2e_fields* f, int where,
                                      int32_t* policy_out, float* value_out, int out_where,
                                      e2e_fused_stats* stats, void* stream) {
  e2e_status vs = validate_problem(p);
  if (vs != E2E_OK) return vs;
  if (!f || !f->u || !f->v || !f->yi || !f->s || !f->mask || (p->nmodes > 0 && (!f->ui || !f->vi)))
    return fail(E2E_ERR_INVALID, "null field pointer");
  if (where != E2E_HOST && where != E2E_DEVICE) return fail(E2E_ERR_INVALID, "bad fields_where");
  if (out_where != E2E_HOST && out_where != E2E_DEVICE) return fail(E2E_ERR_INVALID, "bad out_where");
  cudaStream_t st = (cudaStream_t)stream;

  BuildPlan pl;
  e2e_status s = plan_build(p, 32, 0, &pl);
  if (s != E2E_OK) return s;
  DeviceScratch scratch(st);
  FieldsOnDevice fd;
  s = fields_to_device(p, f, where, st, &fd, &scratch);
  if (s != E2E_OK) return s;
  DevProblem D;
  s = make_dev_problem(p, st, &D, &scratch);
  if (s != E2E_OK) return s;

  const int64_t ns = pl.ns, nc = pl.ncells;
  float* dV = nullptr;
  int32_t* dpi = nullptr;
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
  // the last layer has no rows: value 0 and action 0 (the first of equal
  // zero Q values), as the sweeps give it
  const int64_t last = (int64_t)(p->nt - 1) * nc;
  CK(cudaMemsetAsync(dV + last, 0, sizeof(float) * (size_t)nc, st));
  CK(cudaMemsetAsync(dpi + last, 0, sizeof(int32_t) * (size_t)nc, st));

  unsigned long long* ctr = nullptr;
  CK(dalloc((void**)&ctr, sizeof(unsigned long long) * CTR_COUNT, st));
  scratch.add(ctr);
  unsigned int* done = nullptr;  // per (layer, grid row): cells backed up
  const size_t n_done = (size_t)p->nt * (size_t)p->gsize;
  CK(dalloc((void**)&done, sizeof(unsigned int) * n_done, st));
  scratch.add(done);
  // bound of one wait for a layer's completion: E2E_WAIT_LIMIT_MS (default
  // 5000); E2E_TEST_UNREACHABLE_WAIT=1 raises the targets so that none
  // completes (tests of the bounded waits only)
  unsigned long long wait_ns = 5000000000ull;
  if (const char* ms = std::getenv("E2E_WAIT_LIMIT_MS")) {
    const double v = std::atof(ms);
    if (v > 0 && v <= 60000) wait_ns = (unsigned long long)(v * 1e6);
  }
  const char* unreachable = std::getenv("E2E_TEST_UNREACHABLE_WAIT");
  const unsigned int wait_extra = (unreachable && unreachable[0] == '1') ? 1u : 0u;
  const int mm = p->neighb_gsize * p->neighb_gsize;
  int64_t pool_units = pl.pool_units;
  uint32_t* pool = nullptr;
  unsigned long long hc[CTR_COUNT];
  cudaEvent_t ev[2];
  for (int k = 0; k < 2; ++k) CK(cudaEventCreate(&ev[k]));
  struct EvFree {
    cudaEvent_t* e;
    ~EvFree() { for (int k = 0; k < 2; ++k) cudaEventDestroy(e[k]); }
  } evfree{ev};
  int launches = 0;
  for (int attempt = 0; attempt < 3; ++attempt) {
    if (!pool) CK(dalloc((void**)&pool, sizeof(uint32_t) * (size_t)mm * (size_t)pool_units, st));
    CK(cudaMemsetAsync(ctr, 0, sizeof(unsigned long long) * CTR_COUNT, st));
    CK(cudaMemsetAsync(done, 0, sizeof(unsigned int) * n_done, st));
    BuildArgs A{};
    A.P = D;
    A.F = fd.F;
    A.tiles_per_layer = (int)pl.tiles_per_layer;
    A.rc = pl.rc;
    A.ybufs = pl.ybufs;
    A.lanes_log2 = build_lanes_log2(pl.na);
    A.counters = ctr;
    A.pool = pool;
    A.pool_units = pool_units;
    A.V = dV;
    A.pi = dpi;
    A.layer_done = done;
    A.wait_ns = wait_ns;
    A.wait_extra = wait_extra;
    CK(cudaEventRecord(ev[0], st));
    if (p->nt > 1) {
      int grid = 0;
      CK(launch_build_fused(A, st, &grid));
      ++launches;
    }
    CK(cudaEventRecord(ev[1], st));
    // sleep through the pass, then read its counters
    CK(sleep_sync(st));
    CK(cudaMemcpyAsync(hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hc[CTR_FLAGS] & FLAG_WAIT_TIMEOUT)
      return fail(E2E_ERR_DEVICE, "fused build+backup: a wait for a layer's completion ran out of its bound");
    if (!(hc[CTR_FLAGS] & FLAG_POOL_EXHAUSTED)) break;
    // rows that found no dense histogram were not backed up: again with the
    // pool size the pass asked for
    dfree(pool, st);
    pool = nullptr;
    pool_units = (int64_t)hc[CTR_POOL];
    if ((double)pool_units * mm * 4 > 32.0 * (1ull << 30))
      return fail(E2E_ERR_UNSUPPORTED, "transition spread too wide: dense-histogram pool above 32 GiB");
    if (attempt == 2) return fail(E2E_ERR_DEVICE, "fused build did not settle after re-runs");
  }
  scratch.add(pool);
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
  if (out_where == E2E_HOST) {
    if (value_out) CK(cudaMemcpyAsync(value_out, dV, sizeof(float) * ns, cudaMemcpyDeviceToHost, st));
    if (policy_out) CK(cudaMemcpyAsync(policy_out, dpi, sizeof(int32_t) * ns, cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  if (stats) {
    stats->seconds = ms * 1e-3;
    stats->n_rows = pl.n_rows;
    stats->nnz = (int64_t)hc[CTR_STAGE];
    stats->dropped = hc[CTR_DROPPED];
    stats->misbinned = hc[CTR_MISBIN];
    stats->overflow_rows = hc[CTR_OVERFLOW_ROWS];
    stats->launches = launches;
    stats->h2d_bytes = (int64_t)fd.h2d_bytes;
  }
  return E2E_OK;
}
