// K4: fused sparse value iteration.
//
// The reference's iteration (solver_do_backup + compute_sup_norm,
// src/spvi_2.cu:174-356) makes four passes over memory per sweep:
//   cudaMemcpy Q <- R (:186), cusparseSpMV Q += P V over the COO (:225-234),
//   select_best_action over Q (:93-122, :247) and reduce_sup_norm (:129-171)
//   plus a D2D copy V <- V' (:696).
// Here one kernel does the row sums of every action of a state, the argmax
// (first maximum, start value -1e6 / action -1, as select_best_action) and the
// FP64 sup-norm in a single pass; Q is never materialised and V ping-pongs.
//
// Thread layout: the actions of one state sit in a group of `lanes` (power of
// two >= num_actions) consecutive threads of a warp; each thread reduces one
// row (s, a) of the state-major CSR; the group's argmax is a xor-shuffle tree.
#include <math.h>

#include "kernels.h"

namespace e2e {

template <typename CntT>
__device__ __forceinline__ float load_w(const CntT* __restrict__ c, int64_t k) {
  return to_f(__ldg(c + k));
}

template <typename PtrT, typename CntT>
__global__ void __launch_bounds__(256) k_vi_sweep(ViModel M, int64_t s_begin, int64_t s_end,
                                                  int lanes_log2, const float* Vin, float* Vout,
                                                  int32_t* pi, unsigned long long* resid) {
  const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lanes = 1 << lanes_log2;
  const int a = (int)(gt & (lanes - 1));
  const int64_t s = s_begin + (gt >> lanes_log2);
  const bool in_state = s < s_end;
  const bool act = in_state && a < M.na;
  const bool counts = M.count_type != VAL_F32;
  float q = 0.f;
  bool ok = false;
  if (act) {
    const int64_t row = s * M.na + a;
    q = __ldg(M.R + row);
    if (s < M.n_row_states) {
      const PtrT* __restrict__ rp = reinterpret_cast<const PtrT*>(M.row_ptr);
      const int64_t b = (int64_t)__ldg(rp + row), e = (int64_t)__ldg(rp + row + 1);
      const CntT* __restrict__ cnt = reinterpret_cast<const CntT*>(M.cnt);
      float acc = 0.f;
      for (int64_t k = b; k < e; ++k) acc += load_w(cnt, k) * Vin[__ldg(M.col + k)];
      q = finish_row(q, acc, 0.f, M.nrzns, counts);
    }
    ok = !isnan(q);
  }
  float bq = ok ? q : -INFINITY;
  int ba = ok ? a : 0x7fffffff;
  for (int off = lanes >> 1; off > 0; off >>= 1) {
    float oq = __shfl_xor_sync(0xffffffffu, bq, off);
    int oa = __shfl_xor_sync(0xffffffffu, ba, off);
    if (oq > bq || (oq == bq && oa < ba)) {
      bq = oq;
      ba = oa;
    }
  }
  double d = 0.0;
  if (in_state && a == 0) {
    float vout;
    int32_t pout;
    if (bq > -1e6f) {
      vout = bq;
      pout = ba;
    } else {
      vout = -1e6f;
      pout = -1;
    }
    if (resid) d = fabs((double)vout - (double)Vin[s]);
    Vout[s] = vout;
    pi[s] = pout;
  }
  if (resid) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) d = fmax(d, __shfl_xor_sync(0xffffffffu, d, off));
    __shared__ double wmax[8];
    if ((threadIdx.x & 31) == 0) wmax[threadIdx.x >> 5] = d;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mx = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, wmax[w]);
      if (mx > 0.0) atomicMax(resid, (unsigned long long)__double_as_longlong(mx));
    }
  }
}

template <typename PtrT, typename CntT>
__global__ void __launch_bounds__(256) k_vi_sweep_f64(ViModel M, int64_t s_begin, int64_t s_end,
                                                      int lanes_log2, double* V) {
  const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lanes = 1 << lanes_log2;
  const int a = (int)(gt & (lanes - 1));
  const int64_t s = s_begin + (gt >> lanes_log2);
  const bool in_state = s < s_end;
  const bool act = in_state && a < M.na;
  double q = -INFINITY;
  if (act) {
    const int64_t row = s * M.na + a;
    q = (double)__ldg(M.R + row);
    if (s < M.n_row_states) {
      const PtrT* __restrict__ rp = reinterpret_cast<const PtrT*>(M.row_ptr);
      const int64_t b = (int64_t)__ldg(rp + row), e = (int64_t)__ldg(rp + row + 1);
      const CntT* __restrict__ cnt = reinterpret_cast<const CntT*>(M.cnt);
      double acc = 0.0;
      for (int64_t k = b; k < e; ++k) acc += (double)load_w(cnt, k) * V[__ldg(M.col + k)];
      q = (M.count_type != VAL_F32) ? q + acc / (double)M.nrzns : q + acc;
    }
    if (isnan(q)) q = -INFINITY;
  }
  for (int off = lanes >> 1; off > 0; off >>= 1) q = fmax(q, __shfl_xor_sync(0xffffffffu, q, off));
  if (in_state && a == 0) V[s] = q > -1e6 ? q : -1e6;
}

__global__ void k_compare_f64(const float* V, const double* Vd, int64_t n,
                              unsigned long long* err) {
  double e = 0.0, mref = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    e = fmax(e, fabs((double)V[i] - Vd[i]));
    mref = fmax(mref, fabs(Vd[i]));
  }
  for (int off = 16; off > 0; off >>= 1) {
    e = fmax(e, __shfl_xor_sync(0xffffffffu, e, off));
    mref = fmax(mref, __shfl_xor_sync(0xffffffffu, mref, off));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(err, (unsigned long long)__double_as_longlong(e));
    atomicMax(err + 1, (unsigned long long)__double_as_longlong(mref));
  }
}

static int lanes_log2_for(int na) {
  int l = 0;
  while ((1 << l) < na) ++l;
  return l;
}

template <typename F>
static cudaError_t dispatch(const ViModel& M, F&& f) {
  if (M.index_bits == 32) {
    if (M.count_type == CNT_U16) return f((int32_t*)0, (uint16_t*)0);
    if (M.count_type == CNT_U32) return f((int32_t*)0, (uint32_t*)0);
    return f((int32_t*)0, (float*)0);
  }
  if (M.count_type == CNT_U16) return f((int64_t*)0, (uint16_t*)0);
  if (M.count_type == CNT_U32) return f((int64_t*)0, (uint32_t*)0);
  return f((int64_t*)0, (float*)0);
}

cudaError_t launch_vi_sweep(const ViModel& M, int64_t s_begin, int64_t s_end, const float* Vin,
                            float* Vout, int32_t* pi, unsigned long long* resid,
                            cudaStream_t st) {
  if (s_end <= s_begin) return cudaSuccess;
  const int ll = lanes_log2_for(M.na);
  const int64_t threads = (s_end - s_begin) << ll;
  const unsigned blocks = (unsigned)((threads + 255) / 256);
  return dispatch(M, [&](auto* p, auto* c) {
    using PtrT = std::remove_pointer_t<decltype(p)>;
    using CntT = std::remove_pointer_t<decltype(c)>;
    k_vi_sweep<PtrT, CntT><<<blocks, 256, 0, st>>>(M, s_begin, s_end, ll, Vin, Vout, pi, resid);
    return cudaGetLastError();
  });
}

cudaError_t launch_vi_sweep_f64(const ViModel& M, int64_t s_begin, int64_t s_end, double* V,
                                cudaStream_t st) {
  if (s_end <= s_begin) return cudaSuccess;
  const int ll = lanes_log2_for(M.na);
  const int64_t threads = (s_end - s_begin) << ll;
  const unsigned blocks = (unsigned)((threads + 255) / 256);
  return dispatch(M, [&](auto* p, auto* c) {
    using PtrT = std::remove_pointer_t<decltype(p)>;
    using CntT = std::remove_pointer_t<decltype(c)>;
    k_vi_sweep_f64<PtrT, CntT><<<blocks, 256, 0, st>>>(M, s_begin, s_end, ll, V);
    return cudaGetLastError();
  });
}

cudaError_t launch_compare_f64(const float* V, const double* Vd, int64_t n,
                               unsigned long long* err, cudaStream_t st) {
  k_compare_f64<<<148 * 4, 256, 0, st>>>(V, Vd, n, err);
  return cudaGetLastError();
}

}  // namespace e2e
