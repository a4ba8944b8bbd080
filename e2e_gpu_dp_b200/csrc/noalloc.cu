// e2e_spvi_solve_noalloc: the value-iteration solve without any device
// allocation.
//
// Some callers of this library cannot call cudaMalloc: a serving loop whose
// device memory is already fully reserved by its own pool (an extra allocation
// can fail or fragment that pool), or code running while another framework's
// caching allocator owns the device.  For them this entry point runs the same
// sweep kernel (k_vi_sweep) as e2e_spvi_solve, but its scratch -- the second
// value buffer of the Jacobi ping-pong / the verification sweep, and the
// residual word -- lives in the fixed file-scope device array below.
//
// Limits and sharing:
//  * the array holds one residual word and a value buffer of kNoAllocMaxStates
//    floats; models with more states are rejected with E2E_ERR_UNSUPPORTED.
//    The number of sweeps is not limited: the host reads the residual back
//    after every sweep, so one word, cleared before each sweep, serves them all;
//  * every GPU that loads this library keeps the array (32 MiB) until exit;
//  * all calls share the array and it keeps the last call's contents: each call
//    clears the residual word before every sweep; calls whose work overlaps on
//    the GPU (e.g. concurrent streams) race on the array and must be serialised
//    by the caller;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it for the
//    life of the process; make that first call before any stream capture.  The
//    cached address belongs to the device's primary context: after
//    cudaDeviceReset the process must not call this entry point again;
//  * the layered method's policy comes from its verification sweep (the
//    regular solve reports the layered pass's actions); both are the same
//    whenever every transition of the model leads from layer t to layer t+1,
//    which holds for every model the builder makes.
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <mutex>

#include "e2e_dp.h"
#include "internal.h"
#include "kernels.h"

using namespace e2e;

namespace {

constexpr size_t kNoAllocBytes = size_t(32) << 20;  // 32 MiB
constexpr size_t kNoAllocResidBytes = 256;          // the residual word, padded to the value buffer's alignment
constexpr size_t kNoAllocMaxStates = (kNoAllocBytes - kNoAllocResidBytes) / sizeof(float);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {nullptr};

e2e_status scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(E2E_ERR_UNSUPPORTED, "device index above 63");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return E2E_OK;
}

}  // namespace

// After work has been queued on the shared array, an error return first waits
// for that work, so that a call the caller makes right after the error does
// not race with it.
#define CK(call)                                          \
  do {                                                    \
    cudaError_t _e = (call);                              \
    if (_e != cudaSuccess) {                              \
      cudaStreamSynchronize(st);                          \
      return cuda_fail(_e, #call);                        \
    }                                                     \
  } while (0)

extern "C" e2e_status e2e_spvi_solve_noalloc(const e2e_model* m, const e2e_vi_opts* opts,
                                             int32_t* policy_dev, float* value_dev,
                                             e2e_vi_stats* stats, void* stream) {
  if (!m || !policy_dev || !value_dev) return fail(E2E_ERR_INVALID, "null argument");
  e2e_vi_opts o{};
  o.method = m->layered ? 1 : 0;
  o.threshold = 0.1f;
  if (opts) o = *opts;
  if (o.method != 0 && o.method != 1) return fail(E2E_ERR_INVALID, "method must be 0 or 1");
  if (o.fp64_check) return fail(E2E_ERR_UNSUPPORTED, "fp64_check needs device allocation; use e2e_spvi_solve");
  const int64_t ns = m->ns;
  if ((size_t)ns > kNoAllocMaxStates)
    return fail(E2E_ERR_UNSUPPORTED, "model has " + std::to_string(ns) +
                                         " states; the no-allocation solve holds at most " +
                                         std::to_string(kNoAllocMaxStates));
  if (o.method == 1 && (!m->layered || m->ncells <= 0 || m->nt <= 0))
    return fail(E2E_ERR_UNSUPPORTED, "layered solve needs a time-layered model (nt, ncells known)");
  // the same default as e2e_spvi_solve
  const int max_iter = o.max_iter > 0 ? o.max_iter : (m->nt > 0 ? m->nt + 2 : 100000);
  void* base = nullptr;
  e2e_status s = scratch_address(&base);
  if (s != E2E_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  unsigned long long* resid = reinterpret_cast<unsigned long long*>(base);
  float* W = reinterpret_cast<float*>(static_cast<unsigned char*>(base) + kNoAllocResidBytes);
  const ViModel M = vi_model(m);
  auto t0 = std::chrono::steady_clock::now();
  int iters = 0;
  double last = 0.0;
  e2e_status result = E2E_OK;
  // one sweep that reports its FP64 residual; the word is cleared first since
  // the array keeps whatever the previous sweep or call left there
  auto residual_sweep = [&](const float* vin, float* vout) -> cudaError_t {
    cudaError_t e = cudaMemsetAsync(resid, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    e = launch_vi_sweep(M, 0, ns, vin, vout, policy_dev, resid, st);
    if (e != cudaSuccess) return e;
    unsigned long long h = 0;
    e = cudaMemcpyAsync(&h, resid, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    std::memcpy(&last, &h, sizeof(double));
    return cudaSuccess;
  };
  if (o.method == 1) {
    const int64_t nc = m->ncells;
    CK(launch_vi_sweep(M, m->n_row_states, ns, value_dev, value_dev, policy_dev, nullptr, st));
    for (int64_t t = (m->n_row_states / nc) - 1; t >= 0; --t)
      CK(launch_vi_sweep(M, t * nc, (t + 1) * nc, value_dev, value_dev, policy_dev, nullptr, st));
    // verification sweep: values into the scratch buffer; its actions overwrite
    // the caller's policy with the same actions (same inputs, same arithmetic)
    CK(residual_sweep(value_dev, W));
    iters = 2;
  } else {
    float* a = value_dev;
    float* b = W;
    CK(cudaMemsetAsync(a, 0, sizeof(float) * (size_t)ns, st));
    bool done = false;
    while (!done && iters < max_iter) {
      ++iters;
      CK(residual_sweep(a, b));
      float* tmp = a;
      a = b;
      b = tmp;
      if (last < (double)o.threshold) done = true;
      if (!done && o.timeout_s > 0 &&
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > o.timeout_s) {
        result = fail(E2E_ERR_TIMEOUT, "value iteration exceeded timeout_s");
        break;
      }
    }
    if (a != value_dev)
      CK(cudaMemcpyAsync(value_dev, a, sizeof(float) * (size_t)ns, cudaMemcpyDeviceToDevice, st));
    CK(cudaStreamSynchronize(st));
    if (result == E2E_OK && !done) result = fail(E2E_ERR_NOT_CONVERGED, "max_iter reached before the threshold");
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = iters;
    stats->residual = last;
    stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const int64_t pb = m->index_bits == 32 ? 4 : 8, cb = m->count_type == E2E_COUNT_U16 ? 2 : 4;
    stats->bytes_per_sweep = (m->n_rows + 1) * pb + m->nnz * (4 + cb) + ns * m->na * 4 + ns * 12;
  }
  return result;
}
