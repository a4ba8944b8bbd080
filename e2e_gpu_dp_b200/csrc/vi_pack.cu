// K5 + K6: the sliced copy of a model that value iteration streams, and the
// sweeps over it.
//
// Layout.  States are taken in chunks of 32 consecutive states of one layer
// (a chunk never crosses a layer boundary; the last chunk of a layer is
// partial).  Lane l of a warp owns state l of a chunk.  For action a, a chunk
// stores maxlen[c][a] "slot rows" of 32 entries; entry k of row (s, a) sits at
//   slot (chunk_slot[c] + sum_{b<a} maxlen[c][b] + k) * 32 + lane(s)
// so the k-th entries of the 32 rows (s, a) of a chunk are one coalesced
// 128-byte line.  Rows shorter than maxlen are padded with count 0.  R is
// stored beside it as [chunk][action][lane].
//
// Columns: on a time-layered model built on a g x g grid, every next state of
// a layer-t cell (i, j) lies in layer t+1 inside the m x m window centred on
// (i, j), so it is stored as the 16-bit offset col - base(s) with
//   base(s) = (t+1)*g^2 + (i-del)*g + (j-del),  0 <= offset <= (m-1)(g+1).
// With uint16 counts an entry is one uint32 (offset | count << 16).  Models
// without that geometry keep int32 columns and a separate count array.
//
// Arithmetic.  A row's sum is the same FMA chain in entry order as every
// other solver path of this package (finish_row), followed by fma(0, v, acc)
// for each padding slot, which returns acc unchanged as long as v is finite
// (acc is never -0: it starts at +0 and RN addition gives -0 only from two -0
// operands).  A padding slot therefore points at the lane's own cell in layer
// t+1, whose value is final before layer t is computed in any schedule, never
// at memory the current sweep has not written yet.  Values are bit-identical
// to the CSR sweep.
//
// Per row the sweep reads (offset + count) per padded entry, R, and the
// gathered V; there is no row pointer.  The first-maximum argmax is taken
// in action order inside the lane (the reference's select_best_action,
// src/spvi_2.cu:93-122: start -1e6 / -1, strict '>').
#include <math.h>

#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "internal.h"

namespace e2e {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int PF_NEXT = VI_TUNE_PF_NEXT;
constexpr int PF_CURRENT = VI_TUNE_PF_CURRENT;
constexpr long long kBarrierSpinLimit = 1ll << 22;
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s

// Bounds of the device-side waits of the persistent sweeps (grid barriers of
// the layered sweep, per-layer completion counters of the batched sweep): a
// wait gives up after `spins` polls or `timeout_ns`, sets an error bit the
// host reads (E2E_ERR_DEVICE) and lets the launch drain.  `extra` raises every
// wait's target so that no wait can complete: the test hook that makes the
// bounded waits run out on purpose, without any fault.
struct WaitBound {
  unsigned long long timeout_ns;
  long long spins;
  unsigned int extra;
};

// Host: E2E_WAIT_LIMIT_MS (default 2000) bounds each wait; with
// E2E_TEST_UNREACHABLE_WAIT=1 the targets are raised by one (tests only).
WaitBound wait_bound_from_env() {
  WaitBound w{kBarrierTimeoutNs, kBarrierSpinLimit, 0u};
  if (const char* ms = std::getenv("E2E_WAIT_LIMIT_MS")) {
    const double v = std::atof(ms);
    if (v > 0 && v <= 60000) w.timeout_ns = (unsigned long long)(v * 1e6);
  }
  if (const char* u = std::getenv("E2E_TEST_UNREACHABLE_WAIT")) w.extra = (u[0] == '1') ? 1u : 0u;
  return w;
}

__device__ __forceinline__ void prefetch_l2(const void* p, uint32_t bytes) {
  // bulk prefetch into L2: no shared memory, no completion to wait for
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ld_acquire_s32(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) {
  return __ldcs(p);
}

template <bool COHERENT>
__device__ __forceinline__ float ld_value(const float* p) {
  // V written by other CTAs of the same persistent launch: an ordinary
  // (weak, L1-cached) load, never the read-only path.  Every reader is
  // ordered after an acquire of the completion that released those writes
  // (grid barrier, or its own acquire of the layer counter), so the memory
  // model makes it observe them.
  if (COHERENT) return *p;  // not const __restrict__: the compiler keeps the coherent path
  return __ldg(p);
}

struct ChunkPos {
  int64_t s;      // state of this lane
  int64_t base;   // window base of the lane's columns (window-offset layouts) or 0
  bool valid;     // the lane's state exists
};

// chunk indices, layer sizes and grid sides fit in 32 bits (checked on the host)
__device__ __forceinline__ ChunkPos chunk_pos(const ViPack& P, int c, int lane, bool window) {
  ChunkPos r;
  const int cpl = (int)P.cpl, nc = (int)P.nc;
  const int t = c / cpl;
  const int sl = (c - t * cpl) * 32 + lane;
  r.valid = sl < nc;
  r.s = (int64_t)t * nc + sl;
  r.base = 0;
  if (window && r.valid && r.s < P.n_row_states && t + 1 < P.nlayers) {
    const int i = sl / P.g;
    const int j = sl - i * P.g;
    r.base = (int64_t)(t + 1) * nc + (int64_t)(i - P.del) * P.g + (j - P.del);
  }
  return r;
}

// Entry streams of the three layouts:
//   ENT_PACKED : uint32 per entry, window offset | count << 16
//   ENT_OFF16  : uint16 window offset + count array (uint32 counts / float values)
//   ENT_I32    : int32 column + count array
template <int MODE, typename CntT>
struct Entries {
  using ColT = typename std::conditional<
      MODE == ENT_PACKED, uint32_t,
      typename std::conditional<MODE == ENT_OFF16, uint16_t, int32_t>::type>::type;
  const ColT* col;
  const CntT* cnt;
  __device__ __forceinline__ void advance(int rows) {
    col += rows * 32;
    if (MODE != ENT_PACKED) cnt += rows * 32;
  }
  // this lane's first n (<= B) entries, zeros beyond; a full batch loads unpredicated
  template <int B>
  __device__ __forceinline__ void load(int n, ColT (&o)[B], CntT (&w)[B]) const {
    if (n == B) {
#pragma unroll
      for (int j = 0; j < B; ++j) {
        o[j] = ld_stream(col + j * 32);
        w[j] = MODE != ENT_PACKED ? ld_stream(cnt + j * 32) : (CntT)0;
      }
      return;
    }
#pragma unroll
    for (int j = 0; j < B; ++j) {
      o[j] = 0;
      w[j] = 0;
      if (j < n) {
        o[j] = ld_stream(col + j * 32);
        if (MODE != ENT_PACKED) w[j] = ld_stream(cnt + j * 32);
      }
    }
  }
};

// V index and weight of one entry
template <int MODE, typename ColT, typename CntT>
__device__ __forceinline__ void decode(ColT o, CntT w, uint32_t& idx, float& f) {
  if (MODE == ENT_PACKED) {
    idx = o & 0xffffu;
    f = (float)(o >> 16);
  } else {
    idx = (uint32_t)o;
    f = to_f(w);
  }
}

// The sum over a row's N slots (N = the (chunk, action) slot count, the same
// for the whole warp): every entry load, then every gather, then the fma chain
// in slot order.  Slots past the lane's row hold count 0 and point at a value
// that is finite, so they add fma(0, v, acc) = acc.
template <int N, int MODE, typename CntT, bool COHERENT>
__device__ __forceinline__ float row_slots(const Entries<MODE, CntT>& e, const float* vb) {
  using ColT = typename Entries<MODE, CntT>::ColT;
  ColT o[N];
  CntT w[N];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    o[j] = ld_stream(e.col + j * 32);
    w[j] = MODE != ENT_PACKED ? ld_stream(e.cnt + j * 32) : (CntT)0;
  }
  float v[N], f[N];
#pragma unroll
  for (int j = 0; j < N; ++j) {
    uint32_t idx;
    decode<MODE, ColT, CntT>(o[j], w[j], idx, f[j]);
    v[j] = ld_value<COHERENT>(vb + idx);
  }
  float acc = 0.f;
#pragma unroll
  for (int j = 0; j < N; ++j) acc = fmaf(f[j], v[j], acc);
  return acc;
}

// Best (value, action) over actions [a0, a1) of the lane's state of chunk c;
// the lane's R of action a is Rp[(a - a0) * rstride].  VAR 0: the next
// action's first batch of 4 entries is loaded before this action's gathers
// (5 CTAs per SM).  VAR 1: no look-ahead, fewer registers and 8 CTAs per SM;
// latency is hidden by the extra warps instead.  VAR 2: as VAR 1, but a row of
// up to 10 slots is one straight-line block for its exact slot count (a
// switch on the warp-uniform count) instead of predicated batches of 4.
template <int MODE, typename CntT, bool COHERENT, int VAR>
__device__ __forceinline__ void chunk_best(const ViPack& P, int c, const ChunkPos& cp, int lane, int a0,
                                           int a1, const float* Vin, float& bq, int& ba,
                                           const float* Rp, int rstride) {
  using E = Entries<MODE, CntT>;
  using ColT = typename E::ColT;
  constexpr int B = 4;
  const uint16_t* mlp = P.maxlen + (int64_t)c * P.na_pad;
  int64_t slot = __ldg(P.chunk_slot + c);
  for (int b = 0; b < a0; ++b) slot += __ldg(mlp + b);
  E cur{reinterpret_cast<const ColT*>(P.col) + slot * 32 + lane,
        MODE == ENT_PACKED ? nullptr : reinterpret_cast<const CntT*>(P.cnt) + slot * 32 + lane};
  const float* vb = MODE == ENT_I32 ? Vin : Vin + cp.base;
  const bool counts = P.count_type != VAL_F32;
  auto fold = [&](const ColT(&o)[B], const CntT(&w)[B], int n, float& acc) {
    float v[B], f[B];
#pragma unroll
    for (int j = 0; j < B; ++j) {
      uint32_t idx;
      decode<MODE, ColT, CntT>(o[j], w[j], idx, f[j]);
      v[j] = j < n ? ld_value<COHERENT>(vb + idx) : 0.f;
    }
    // entries beyond n hold count 0 and v = 0: fma(0, 0, acc) == acc
#pragma unroll
    for (int j = 0; j < B; ++j) acc = fmaf(f[j], v[j], acc);
  };
  if constexpr (VAR == 2) {
    for (int a = a0; a < a1; ++a) {
      const float r = ld_stream(Rp);
      Rp += rstride;
      const int ml = __ldg(mlp + a);
      float acc = 0.f;
      switch (ml) {
        case 0: break;
        case 1: acc = row_slots<1, MODE, CntT, COHERENT>(cur, vb); break;
        case 2: acc = row_slots<2, MODE, CntT, COHERENT>(cur, vb); break;
        case 3: acc = row_slots<3, MODE, CntT, COHERENT>(cur, vb); break;
        case 4: acc = row_slots<4, MODE, CntT, COHERENT>(cur, vb); break;
        case 5: acc = row_slots<5, MODE, CntT, COHERENT>(cur, vb); break;
        case 6: acc = row_slots<6, MODE, CntT, COHERENT>(cur, vb); break;
        case 7: acc = row_slots<7, MODE, CntT, COHERENT>(cur, vb); break;
        case 8: acc = row_slots<8, MODE, CntT, COHERENT>(cur, vb); break;
        case 9: acc = row_slots<9, MODE, CntT, COHERENT>(cur, vb); break;
        case 10: acc = row_slots<10, MODE, CntT, COHERENT>(cur, vb); break;
        default:
          for (int k0 = 0; k0 < ml; k0 += B) {
            E more = cur;
            more.advance(k0);
            ColT o2[B];
            CntT w2[B];
            more.template load<B>(min(ml - k0, B), o2, w2);
            fold(o2, w2, min(ml - k0, B), acc);
          }
      }
      const float q = finish_row(r, acc, 0.f, P.nrzns, counts);
      if (!isnan(q) && q > bq) {
        bq = q;
        ba = a;
      }
      cur.advance(ml);
    }
    return;
  }
  int ml = a0 < a1 ? __ldg(mlp + a0) : 0;
  ColT o[B];
  CntT w[B];
  if (VAR == 0) cur.template load<B>(min(ml, B), o, w);
  for (int a = a0; a < a1; ++a) {
    const float r = ld_stream(Rp);
    Rp += rstride;
    float acc = 0.f;
    int mln = 0;
    E nxt = cur;
    nxt.advance(ml);
    if (VAR == 0) {
      mln = a + 1 < a1 ? __ldg(mlp + a + 1) : 0;
      ColT no[B];
      CntT nw[B];
      nxt.template load<B>(min(mln, B), no, nw);
      fold(o, w, min(ml, B), acc);
#pragma unroll
      for (int j = 0; j < B; ++j) {
        o[j] = no[j];
        w[j] = nw[j];
      }
    } else {
      cur.template load<B>(min(ml, B), o, w);
      fold(o, w, min(ml, B), acc);
    }
    for (int k0 = B; k0 < ml; k0 += B) {  // rows longer than one batch
      E more = cur;
      more.advance(k0);
      ColT o2[B];
      CntT w2[B];
      more.template load<B>(min(ml - k0, B), o2, w2);
      fold(o2, w2, min(ml - k0, B), acc);
    }
    const float q = finish_row(r, acc, 0.f, P.nrzns, counts);
    if (!isnan(q) && q > bq) {
      bq = q;
      ba = a;
    }
    cur = nxt;
    if (VAR == 0) ml = mln;
    else ml = a + 1 < a1 ? __ldg(mlp + a + 1) : 0;
  }
}

// R of (lane's state, action a0) in the pack's [chunk][action][lane] table
__device__ __forceinline__ const float* pack_r(const ViPack& P, int c, int a0, int lane) {
  return P.R + ((int64_t)c * P.na + a0) * 32 + lane;
}

template <int MODE, int VAR>
struct MinBlocks {
  static constexpr int value = MODE != ENT_PACKED ? 3 : (VAR == 0 ? 5 : 8);
};

template <int MODE, typename CntT>
struct Widths {
  static constexpr int col = MODE == ENT_OFF16 ? 2 : 4;
  static constexpr int cnt = MODE == ENT_PACKED ? 0 : (int)sizeof(CntT);
};

// L2 prefetch of chunk c: entry streams and R (bulk prefetch, one lane)
__device__ __forceinline__ void prefetch_chunk(const ViPack& P, int c, int col_bytes, int cnt_bytes) {
  const int64_t s0 = __ldg(P.chunk_slot + c), s1 = __ldg(P.chunk_slot + c + 1);
  const int64_t n = (s1 - s0) * 32;
  if (n > 0) {
    prefetch_l2(reinterpret_cast<const char*>(P.col) + s0 * 32 * col_bytes, (uint32_t)(n * col_bytes));
    if (cnt_bytes)
      prefetch_l2(reinterpret_cast<const char*>(P.cnt) + s0 * 32 * cnt_bytes, (uint32_t)(n * cnt_bytes));
  }
  prefetch_l2(P.R + (int64_t)c * P.na * 32, (uint32_t)(P.na * 32 * 4));
}

__device__ __forceinline__ void finish_state(float bq, int ba, float& vout, int32_t& pout) {
  if (bq > -1e6f) {
    vout = bq;
    pout = ba;
  } else {
    vout = -1e6f;
    pout = -1;
  }
}

// One Jacobi sweep over chunks [c_begin, c_end): warp per chunk, grid-stride;
// prefetch bits: PF_NEXT = the warp's next chunk, PF_CURRENT = the chunk it starts.
template <int MODE, typename CntT, int VAR>
__global__ void __launch_bounds__(kThreads, MinBlocks<MODE, VAR>::value)
    k_vi_chunks(ViPack P, int c_begin, int c_end, const float* __restrict__ Vin, float* Vout, int32_t* pi,
                unsigned long long* resid, int prefetch) {
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * kWarps;
  double dmax = 0.0;
  for (int c = c_begin + blockIdx.x * kWarps + (threadIdx.x >> 5); c < c_end; c += nw) {
    if ((prefetch & PF_NEXT) && lane == 0 && c + nw < c_end)
      prefetch_chunk(P, c + nw, Widths<MODE, CntT>::col, Widths<MODE, CntT>::cnt);
    if ((prefetch & PF_CURRENT) && lane == 0)
      prefetch_chunk(P, c, Widths<MODE, CntT>::col, Widths<MODE, CntT>::cnt);
    const ChunkPos cp = chunk_pos(P, c, lane, MODE != ENT_I32);
    float bq = -INFINITY;
    int ba = 0x7fffffff;
    chunk_best<MODE, CntT, false, VAR>(P, c, cp, lane, 0, P.na, Vin, bq, ba, pack_r(P, c, 0, lane), 32);
    if (cp.valid) {
      float vout;
      int32_t pout;
      finish_state(bq, ba, vout, pout);
      if (resid) dmax = fmax(dmax, fabs((double)vout - (double)Vin[cp.s]));
      Vout[cp.s] = vout;
      pi[cp.s] = pout;
    }
  }
  if (resid) {
    for (int off = 16; off > 0; off >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
    __shared__ double wmax[kWarps];
    if (lane == 0) wmax[threadIdx.x >> 5] = dmax;
    __syncthreads();
    if (threadIdx.x == 0) {
      double mx = 0.0;
      for (int w = 0; w < kWarps; ++w) mx = fmax(mx, wmax[w]);
      if (mx > 0.0) atomicMax(resid, (unsigned long long)__double_as_longlong(mx));
    }
  }
}

// ---- TMA-staged Jacobi sweep (packed layout) ---------------------------------------
// A CTA walks super-chunks of SC consecutive chunks; their entries, R and
// per-action lengths are contiguous ranges of the sliced copy, so one thread
// stages super-chunks NST-1 ahead with three 1-D bulk copies each
// (cp.async.bulk, completion counted on an mbarrier per stage) into a ring of
// NST shared-memory stages while the CTA computes: 8/SC warps per chunk,
// each a block of actions, reading entries from shared memory
// (conflict-free: lane l reads word l of a slot row) and gathering V through
// L1.  DRAM latency is covered by the double buffer instead of by resident
// warps.  A super-chunk whose entries exceed a stage is read from global
// memory.  Waits are bounded (error bit 8 of err).
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// 1-D bulk copy global -> this CTA's shared memory (no multicast); 16-byte
// aligned addresses, size a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

template <int SC>
__host__ __device__ __forceinline__ int sc_r_bytes(int na) { return SC * na * 32 * 4; }
template <int SC>
__host__ __device__ __forceinline__ int sc_ml_bytes(int na_pad) { return (SC * na_pad * 2 + 15) & ~15; }
template <int SC, int EB>
__host__ __device__ __forceinline__ int sc_stage_bytes(int na, int na_pad) {
  return EB + sc_r_bytes<SC>(na) + sc_ml_bytes<SC>(na_pad);
}

template <int SC, int NST, int EB>
__global__ void __launch_bounds__(kThreads)
    k_vi_tma(ViPack P, int c_begin, int c_end, const float* __restrict__ Vin, float* Vout, int32_t* pi,
             unsigned long long* resid, unsigned int* err) {
  constexpr int kScChunks = SC;
  constexpr int kScG = kWarps / SC;
  constexpr int kScEntBytes = EB;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bar[NST];
  __shared__ int s_ok, s_direct[NST];
  __shared__ float sq[kWarps][32];
  __shared__ int sa[kWarps][32];
  __shared__ double wmax[kWarps];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int na = P.na, na_pad = P.na_pad;
  const int stage_bytes = sc_stage_bytes<SC, EB>(na, na_pad);
  const int n_sc = (c_end - c_begin + kScChunks - 1) / kScChunks;
  const int cc = wid / kScG, grp = wid % kScG;
  const int apg = (na + kScG - 1) / kScG;
  const int a0 = min(na, grp * apg), a1 = min(na, a0 + apg);
  const bool counts = P.count_type != VAL_F32;

  auto issue = [&](int sc, int st) {  // thread 0
    const int c0 = c_begin + sc * kScChunks, c1 = min(c0 + kScChunks, c_end);
    const int64_t e0 = __ldg(P.chunk_slot + c0), e1 = __ldg(P.chunk_slot + c1);
    const int64_t eb = (e1 - e0) * 128;
    unsigned char* sp = smem + st * stage_bytes;
    if (eb > kScEntBytes) {  // too large for a stage: read from global memory
      s_direct[st] = 1;
      mbar_expect_tx(&bar[st], 0);
      return;
    }
    s_direct[st] = 0;
    const uint32_t rb = (uint32_t)((c1 - c0) * na * 128);
    const uint32_t mb = (uint32_t)((c1 - c0) * na_pad * 2);
    mbar_expect_tx(&bar[st], (uint32_t)eb + rb + mb);
    if (eb) bulk_g2s(sp, reinterpret_cast<const char*>(P.col) + e0 * 128, (uint32_t)eb, &bar[st]);
    bulk_g2s(sp + kScEntBytes, P.R + (int64_t)c0 * na * 32, rb, &bar[st]);
    bulk_g2s(sp + kScEntBytes + sc_r_bytes<SC>(na), P.maxlen + (int64_t)c0 * na_pad, mb, &bar[st]);
  };

  if (tid == 0) {
    for (int q = 0; q < NST; ++q) mbar_init(&bar[q], 1);
    fence_mbar_init();
  }
  __syncthreads();
  int sc = blockIdx.x;
  if (tid == 0)
    for (int q = 0; q < NST - 1; ++q)
      if (sc + q * (int)gridDim.x < n_sc) issue(sc + q * gridDim.x, q);
  double dmax = 0.0;
  bool failed = false;
  for (int k = 0; sc < n_sc; ++k, sc += gridDim.x) {
    const int st = k % NST;
    if (tid == 0) {
      const int ahead = sc + (NST - 1) * (int)gridDim.x;
      if (ahead < n_sc) {
        fence_proxy_async();  // that stage was read through the generic proxy
        issue(ahead, (k + NST - 1) % NST);
      }
      long long it = 0;
      const uint32_t parity = (uint32_t)((k / NST) & 1);
      while (!mbar_try_wait(&bar[st], parity) && ++it < (1ll << 24)) {
      }
      s_ok = it < (1ll << 24);
    }
    __syncthreads();
    if (!s_ok) {
      if (tid == 0) atomicOr(err, 8u);
      failed = true;
      break;
    }
    const int c0 = c_begin + sc * kScChunks;
    const int c = c0 + cc;
    const bool active = c < c_end;
    float bq = -INFINITY;
    int ba = 0x7fffffff;
    ChunkPos cp{0, 0, false};
    if (active) {
      cp = chunk_pos(P, c, lane, true);
      if (s_direct[st]) {
        chunk_best<ENT_PACKED, uint16_t, false, 1>(P, c, cp, lane, a0, a1, Vin, bq, ba, pack_r(P, c, a0, lane), 32);
      } else {
        const unsigned char* sp = smem + st * stage_bytes;
        const uint32_t* ent = reinterpret_cast<const uint32_t*>(sp);
        const float* Rs = reinterpret_cast<const float*>(sp + kScEntBytes);
        const uint16_t* mls = reinterpret_cast<const uint16_t*>(sp + kScEntBytes + sc_r_bytes<SC>(na)) + cc * na_pad;
        int64_t slot = __ldg(P.chunk_slot + c) - __ldg(P.chunk_slot + c0);
        for (int b = 0; b < a0; ++b) slot += mls[b];
        const uint32_t* ep = ent + slot * 32 + lane;
        const float* rp = Rs + ((int64_t)cc * na + a0) * 32 + lane;
        const float* vb = Vin + cp.base;
        for (int a = a0; a < a1; ++a) {
          const int ml = mls[a];
          float acc = 0.f;
          for (int k0 = 0; k0 < ml; k0 += 4) {
            const int n = min(ml - k0, 4);
            uint32_t e[4];
            float v[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) e[j] = j < n ? ep[(k0 + j) * 32] : 0u;
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = j < n ? __ldg(vb + (e[j] & 0xffffu)) : 0.f;
#pragma unroll
            for (int j = 0; j < 4; ++j) acc = fmaf((float)(e[j] >> 16), v[j], acc);  // padding: exact no-op
          }
          ep += ml * 32;
          const float q = finish_row(*rp, acc, 0.f, P.nrzns, counts);
          rp += 32;
          if (!isnan(q) && q > bq) {
            bq = q;
            ba = a;
          }
        }
      }
    }
    sq[wid][lane] = bq;
    sa[wid][lane] = ba;
    __syncthreads();  // candidates in place; the stage is consumed
    if (active && grp == 0) {
      for (int g2 = 1; g2 < kScG; ++g2) {
        const float oq = sq[wid + g2][lane];
        if (oq > bq) {  // later groups hold later actions: strict '>' keeps the first maximum
          bq = oq;
          ba = sa[wid + g2][lane];
        }
      }
      if (cp.valid) {
        float vout;
        int32_t pout;
        finish_state(bq, ba, vout, pout);
        if (resid) dmax = fmax(dmax, fabs((double)vout - (double)Vin[cp.s]));
        Vout[cp.s] = vout;
        pi[cp.s] = pout;
      }
    }
    __syncthreads();  // sq/sa free for the next super-chunk
  }
  if (failed && tid == 0) {
    // give the copies in flight time to land before the CTA exits
    for (int st = 0; st < NST; ++st) {
      long long it = 0;
      while (!mbar_try_wait(&bar[st], 0) && !mbar_try_wait(&bar[st], 1) && ++it < (1ll << 24)) {
      }
    }
  }
  if (resid) {
    for (int off = 16; off > 0; off >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, off));
    if (lane == 0) wmax[wid] = dmax;
    __syncthreads();
    if (tid == 0) {
      double mx = 0.0;
      for (int w = 0; w < kWarps; ++w) mx = fmax(mx, wmax[w]);
      if (mx > 0.0) atomicMax(resid, (unsigned long long)__double_as_longlong(mx));
    }
  }
}

// Grid-wide barrier of a cooperative launch.  sync[0] counts arrivals (never
// reset inside a launch); a wait that outlives its limit sets bit 1 of sync[1]
// and every later barrier returns false at once.
__device__ __forceinline__ bool grid_barrier(unsigned int* sync, unsigned int target, const WaitBound& wb) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int good = 1;
    __threadfence();
    atomicAdd(sync, 1u);
    const unsigned long long t0 = global_ns();
    long long it = 0;
    while (ld_acquire(sync) < target + wb.extra) {
      if (ld_acquire(sync + 1) != 0u || ++it > wb.spins || global_ns() - t0 > wb.timeout_ns) {
        atomicOr(sync + 1, 2u);
        good = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// The layered (backward-induction) schedule in one persistent launch: layer
// nlayers-1 first (V = max_a R), then layers down to 0, each reading the V of
// the layer after it, with a grid barrier between layers.  `groups` warps
// share a chunk, each taking a contiguous block of actions; their candidates
// are combined in action order through shared memory.  With PF_NEXT, each
// chunk's data for the next layer is prefetched into L2 before this layer's
// work, so HBM streams layer t-1 while layer t computes.
template <int MODE, typename CntT, int VAR>
__global__ void __launch_bounds__(kThreads, MinBlocks<MODE, VAR>::value)
    k_vi_layered(ViPack P, int groups, float* V, int32_t* pi, unsigned int* sync, int prefetch, WaitBound wb) {
  __shared__ float sq[kWarps][32];
  __shared__ int sa[kWarps][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int cpc = kWarps / groups;  // chunks per CTA iteration
  const int grp = wid % groups, slot_in_cta = wid / groups;
  const int apg = (P.na + groups - 1) / groups;
  const int a0 = min(P.na, grp * apg), a1 = min(P.na, a0 + apg);
  const int cpl = (int)P.cpl;
  unsigned int gen = 0;
  for (int t = P.nlayers - 1; t >= 0; --t) {
    for (int b = blockIdx.x * cpc; b < cpl; b += gridDim.x * cpc) {
      const int cc = b + slot_in_cta;
      const bool active = cc < cpl;
      float bq = -INFINITY;
      int ba = 0x7fffffff;
      ChunkPos cp{0, 0, false};
      if (active) {
        const int c = t * cpl + cc;
        if ((prefetch & PF_NEXT) && lane == 0 && grp == 0 && t > 0)
          prefetch_chunk(P, c - cpl, Widths<MODE, CntT>::col, Widths<MODE, CntT>::cnt);
        cp = chunk_pos(P, c, lane, MODE != ENT_I32);
        chunk_best<MODE, CntT, true, VAR>(P, c, cp, lane, a0, a1, V, bq, ba, pack_r(P, c, a0, lane), 32);
      }
      if (groups > 1) {
        sq[wid][lane] = bq;
        sa[wid][lane] = ba;
        __syncthreads();
        if (active && grp == 0) {
          for (int g2 = 1; g2 < groups; ++g2) {
            const float oq = sq[wid + g2][lane];
            if (oq > bq) {  // later groups hold later actions: strict '>' keeps the first maximum
              bq = oq;
              ba = sa[wid + g2][lane];
            }
          }
        }
        __syncthreads();
      }
      if (active && grp == 0 && cp.valid) {
        float vout;
        int32_t pout;
        finish_state(bq, ba, vout, pout);
        V[cp.s] = vout;
        pi[cp.s] = pout;
      }
    }
    if (t > 0) {
      ++gen;
      if (!grid_barrier(sync, gen * gridDim.x, wb)) return;
    }
  }
}

// Many layered solves in one persistent launch.  Step k covers layer
// nlayers-1-k of every job that has more than k layers (jobs sorted by layer
// count, so those are a prefix and their chunks a contiguous item range).
// There is no grid-wide barrier: a chunk of layer t waits only until its own
// job's layer t+1 is complete (done[job][t+1] == chunks per layer), and each
// finished chunk adds one to done[job][t].  Every CTA takes its items in step
// order and all CTAs are resident (cooperative launch), so each wait is for
// items of an earlier step that are finished or running; the waits are
// bounded and a timeout sets bit 2 of err and lets the rest drain quickly.
// Jobs with a target take R of the
// cells around it from their Rwin table, and the target's own cells are
// terminal: the reference leaves such a sample in place with reward 0
// (src/build_model.cu:523-545), i.e. one entry (the cell at t+1, count
// nrzns) and R = 0, evaluated here with the same operations as that row.
template <int MODE, int VAR>
struct BatchMinBlocks {  // the job lookup needs more registers than k_vi_layered (lean, batches of 4:
                        // 6 CTAs per SM measured 24.1 ms on the 256-model batch, 5: 24.7, 8: 25.5;
                        // with exact-count rows and the prefix sums in shared memory 6 CTAs 21.1 ms,
                        // 5 CTAs 19.9 ms, and 3.8 against 4.2 ms for one 300x300x150 job)
  static constexpr int value = MODE != ENT_PACKED ? 3 : (VAR == 0 ? 4 : 5);
};

template <int MODE, typename CntT, int VAR>
__global__ void __launch_bounds__(kThreads, BatchMinBlocks<MODE, VAR>::value)
    k_vi_batch(const unsigned char* table, int job_cap, int groups, int* done, int layer_cap,
               unsigned int* err, int prefetch, WaitBound wb) {
  __shared__ float sq[kWarps][32];
  __shared__ int sa[kWarps][32];
  // the jobs' chunk prefix sums, the same at every step (a step uses a prefix
  // of the jobs): searched in shared memory for every item instead of through
  // eight dependent global loads (batched sweep of 256 models 22.1 -> 21.1 ms)
  __shared__ int cum[kViBatchJobCap + 1];
  const ViBatchHeader* H = reinterpret_cast<const ViBatchHeader*>(table);
  const ViJob* jobs = reinterpret_cast<const ViJob*>(table + kViBatchJobsOffset);
  const int* gcum = reinterpret_cast<const int*>(jobs + job_cap);
  const int* nact = gcum + job_cap + 1;
  for (int i = threadIdx.x; i <= H->njobs; i += blockDim.x) cum[i] = gcum[i];
  __syncthreads();
  const int L = H->max_layers;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int cpc = kWarps / groups;
  const int grp = wid % groups, slot_in_cta = wid / groups;
  for (int k = 0; k < L; ++k) {
    const int nj = nact[k];
    const int n_items = cum[nj];
    for (int b = blockIdx.x * cpc; b < n_items; b += gridDim.x * cpc) {
      const int item = b + slot_in_cta;
      const bool active = item < n_items;
      float bq = -INFINITY;
      int ba = 0x7fffffff;
      bool valid = false;
      float* Vout = nullptr;
      int32_t* pout = nullptr;
      int64_t s_out = 0;
      int* done_slot = nullptr;
      bool skip = false;
      if (active) {
        int lo = 0, hi = nj - 1;  // last job with cum[job] <= item
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (cum[mid] <= item) lo = mid;
          else hi = mid - 1;
        }
        const ViJob& J = jobs[lo];
        const ViPack& P = J.P;
        const int na = P.na;
        const int apg = (na + groups - 1) / groups;
        int a0 = min(na, grp * apg);
        const int a1 = min(na, a0 + apg);
        const int cpl = (int)P.cpl, nc = (int)P.nc;
        const int t = P.nlayers - 1 - k;
        const int c = t * cpl + (item - cum[lo]);
        done_slot = done + (int64_t)lo * layer_cap + t;
        if ((prefetch & PF_NEXT) && lane == 0 && grp == 0 && t > 0)
          prefetch_chunk(P, c - cpl, Widths<MODE, CntT>::col, Widths<MODE, CntT>::cnt);
        if (t + 1 < P.nlayers) {  // layer t+1 of this job complete
          const int* dep = done_slot + 1;
          int ok = 1;
          if (lane == 0) {
            const unsigned long long t0 = global_ns();
            long long it = 0;
            while (ld_acquire_s32(dep) < cpl + (int)wb.extra) {
              if (ld_acquire(err) != 0u || ++it > wb.spins || global_ns() - t0 > wb.timeout_ns) {
                atomicOr(err, 4u);
                ok = 0;
                break;
              }
              __nanosleep(64);
            }
          }
          ok = __shfl_sync(0xffffffffu, ok, 0);
          (void)ld_acquire_s32(dep);  // every lane orders its reads after the producers' writes
          if (!ok) {
            skip = true;  // give up this chunk: nothing computed, nothing written
            a0 = a1;
          }
        }
        const ChunkPos cp = chunk_pos(P, c, lane, MODE != ENT_I32);
        const float* Rp = pack_r(P, c, a0, lane);
        int rstride = 32;
        bool terminal = false;
        if (J.Rwin && cp.valid && t + 1 < P.nlayers) {
          const int sl = (int)(cp.s - (int64_t)t * nc);
          const int i = sl / P.g, j = sl - (sl / P.g) * P.g;
          terminal = i >= J.ti && i < J.ti + J.tsg && j >= J.tj && j < J.tj + J.tsg;
          const int wi = i - J.wi0, wj = j - J.wj0;
          if (wi >= 0 && wi < J.wh && wj >= 0 && wj < J.ww) {
            Rp = J.Rwin + (((int64_t)t * J.wh + wi) * J.ww + wj) * na + a0;
            rstride = 1;
          }
        }
        chunk_best<MODE, CntT, true, VAR>(P, c, cp, lane, a0, a1, J.V, bq, ba, Rp, rstride);
        if (terminal) {
          const float v = ld_value<true>(J.V + cp.s + nc);  // the same cell, layer t+1
          const float acc = fmaf((float)P.nrzns, v, 0.f);
          const float q = finish_row(0.f, acc, 0.f, P.nrzns, true);
          bq = -INFINITY;
          ba = 0x7fffffff;
          if (a0 < a1 && !isnan(q)) {
            bq = q;
            ba = a0;
          }
        }
        valid = cp.valid && !skip;
        Vout = J.V;
        pout = J.pi;
        s_out = cp.s;
      }
      if (groups > 1) {
        sq[wid][lane] = bq;
        sa[wid][lane] = ba;
        __syncthreads();
        if (active && grp == 0) {
          for (int g2 = 1; g2 < groups; ++g2) {
            const float oq = sq[wid + g2][lane];
            if (oq > bq) {  // later groups hold later actions: strict '>' keeps the first maximum
              bq = oq;
              ba = sa[wid + g2][lane];
            }
          }
        }
        __syncthreads();
      }
      if (active && grp == 0) {
        if (valid) {
          float vout;
          int32_t po;
          finish_state(bq, ba, vout, po);
          Vout[s_out] = vout;
          pout[s_out] = po;
        }
        __syncwarp();
        if (lane == 0) {
          __threadfence();  // this chunk's values before its completion count
          atomicAdd(done_slot, 1);
        }
      }
    }
  }
}

// ---- pack construction ------------------------------------------------------------

// per chunk: maxlen of every action over the chunk's 32 rows, and their sum
template <typename PtrT>
__global__ void __launch_bounds__(kThreads) k_pack_count(ViModel M, ViPack P, int32_t* slot_len,
                                                         uint16_t* maxlen) {
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * kWarps + (threadIdx.x >> 5);
  if (c >= P.nchunks) return;
  const ChunkPos cp = chunk_pos(P, c, lane, false);
  const bool has = cp.valid && cp.s < P.n_row_states;
  const PtrT* rp = reinterpret_cast<const PtrT*>(M.row_ptr);
  int64_t prev = has ? (int64_t)rp[cp.s * P.na] : 0;
  int total = 0;
  for (int a = 0; a < P.na; ++a) {
    unsigned len = 0;
    if (has) {
      const int64_t nx = (int64_t)rp[cp.s * P.na + a + 1];
      len = (unsigned)(nx - prev);
      prev = nx;
    }
    const unsigned ml = __reduce_max_sync(0xffffffffu, len);
    if (lane == 0) maxlen[(int64_t)c * P.na_pad + a] = (uint16_t)ml;
    total += (int)ml;
  }
  if (lane == 0) {
    for (int a = P.na; a < P.na_pad; ++a) maxlen[(int64_t)c * P.na_pad + a] = 0;
    slot_len[c] = total;
  }
}

// scatter the CSR rows into the chunk layout; flags[0] |= 1 when a window
// offset does not fit 16 bits (the caller then packs with int32 columns)
template <typename PtrT, int MODE, typename CntT>
__global__ void __launch_bounds__(kThreads) k_pack_fill(ViModel M, ViPack P, void* colv, CntT* cnt,
                                                        float* Rp, unsigned int* flags) {
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * kWarps + (threadIdx.x >> 5);
  if (c >= P.nchunks) return;
  const ChunkPos cp = chunk_pos(P, c, lane, MODE != ENT_I32);
  const bool has = cp.valid && cp.s < P.n_row_states;
  const PtrT* rp = reinterpret_cast<const PtrT*>(M.row_ptr);
  const CntT* src = reinterpret_cast<const CntT*>(M.cnt);
  int64_t slot = P.chunk_slot[c];
  bool bad = false;
  // lanes without rows gather nothing that is kept; give them a valid index too
  const int32_t pad_col = !has ? 0 : (int32_t)(cp.s / P.nc + 1 < P.nlayers ? cp.s + P.nc : cp.s);
  for (int a = 0; a < P.na; ++a) {
    const int ml = P.maxlen[(int64_t)c * P.na_pad + a];
    int64_t rs = 0, len = 0;
    if (has) {
      rs = (int64_t)rp[cp.s * P.na + a];
      len = (int64_t)rp[cp.s * P.na + a + 1] - rs;
    }
    for (int k = 0; k < ml; ++k) {
      const int64_t e = (slot + k) * 32 + lane;
      // padding (count 0) points at the lane's own cell in layer t+1, finished
      // before layer t in every schedule, so the gathered value is finite and
      // fma(0, v, acc) leaves acc unchanged
      int32_t col = pad_col;
      CntT w = 0;
      if (k < len) {
        col = M.col[rs + k];
        w = src[rs + k];
      }
      if (MODE == ENT_I32) {
        reinterpret_cast<int32_t*>(colv)[e] = col;
        cnt[e] = w;
      } else {
        int64_t o = (int64_t)col - cp.base;
        if (o < 0 || o > 65535) {
          bad = true;
          o = 0;
        }
        if (MODE == ENT_PACKED) {
          reinterpret_cast<uint32_t*>(colv)[e] = (uint32_t)o | ((uint32_t)w << 16);
        } else {
          reinterpret_cast<uint16_t*>(colv)[e] = (uint16_t)o;
          cnt[e] = w;
        }
      }
    }
    slot += ml;
    Rp[((int64_t)c * P.na + a) * 32 + lane] = cp.valid ? M.R[cp.s * P.na + a] : 0.f;
  }
  if (bad) atomicOr(flags, 1u);
}

// f(layout constant, count type pointer)
template <typename F>
cudaError_t dispatch_pack(const ViPack& P, F&& f) {
  using Pk = std::integral_constant<int, ENT_PACKED>;
  using O16 = std::integral_constant<int, ENT_OFF16>;
  using I32 = std::integral_constant<int, ENT_I32>;
  switch (P.ent_mode) {
    case ENT_PACKED:
      return f(Pk{}, (uint16_t*)nullptr);
    case ENT_OFF16:
      if (P.count_type == CNT_U32) return f(O16{}, (uint32_t*)nullptr);
      if (P.count_type == VAL_F32) return f(O16{}, (float*)nullptr);
      return cudaErrorInvalidValue;
    default:
      if (P.count_type == CNT_U16) return f(I32{}, (uint16_t*)nullptr);
      if (P.count_type == CNT_U32) return f(I32{}, (uint32_t*)nullptr);
      return f(I32{}, (float*)nullptr);
  }
}

int sm_count_pack() {
  static int n = 0;
  if (n == 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}

int col_bytes_of(const ViPack& P) { return P.ent_mode == ENT_OFF16 ? 2 : 4; }
int cnt_bytes_of(const ViPack& P) {
  return P.ent_mode == ENT_PACKED ? 0 : (P.count_type == CNT_U16 ? 2 : 4);
}

int occupancy(const void* kern) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, 0) != cudaSuccess) return 1;
  return std::max(per_sm, 1);
}

}  // namespace

void free_pack(PackStore* p) {
  if (!p) return;
  for (void*& b : p->bufs) {
    dfree(b, 0);
    b = nullptr;
  }
}

int64_t pack_sweep_bytes(const ViPack& P) {
  // entries (with padding) + R + chunk tables + V read + V' and policy written
  return P.slot_rows * 32 * (col_bytes_of(P) + cnt_bytes_of(P)) + P.nchunks * P.na * 32 * 4 +
         P.nchunks * (8 + P.na_pad * 2) + P.ns * 12;
}

cudaError_t build_pack(const ViModel& M, int64_t nc, int g, int del, PackStore* out, cudaStream_t st) {
  *out = PackStore{};
  ViPack& P = out->v;
  P.ns = M.ns;
  P.nc = (nc > 0 && M.ns % nc == 0) ? nc : M.ns;
  P.nlayers = (int)(M.ns / P.nc);
  P.cpl = (P.nc + 31) / 32;
  P.nchunks = P.cpl * P.nlayers;
  if (P.nc >= ((int64_t)1 << 31) - 64 || P.nchunks >= ((int64_t)1 << 31) - 1)
    return cudaErrorInvalidValue;  // 32-bit chunk arithmetic
  P.n_row_states = M.n_row_states;
  P.na = M.na;
  P.na_pad = (M.na + 7) & ~7;
  P.nrzns = M.nrzns;
  P.count_type = M.count_type;
  P.g = g;
  P.del = del;
  const bool window =
      P.nlayers > 1 && g > 0 && (int64_t)g * g == P.nc && (int64_t)(2 * del) * (g + 1) <= 65535;
  P.ent_mode = !window ? ENT_I32 : (M.count_type == CNT_U16 ? ENT_PACKED : ENT_OFF16);

  cudaError_t e;
  int32_t* slot_len = nullptr;
  int64_t* block_sums = nullptr;
  unsigned int* flags = nullptr;
  auto cleanup = [&]() {
    dfree(slot_len, st);
    dfree(block_sums, st);
    dfree(flags, st);
  };
  const int64_t nb = (P.nchunks + 1023) / 1024 + 1;
  if ((e = dalloc(&out->bufs[0], sizeof(int64_t) * (P.nchunks + 1), st)) != cudaSuccess) return e;
  if ((e = dalloc(&out->bufs[1], sizeof(uint16_t) * P.nchunks * P.na_pad, st)) != cudaSuccess) return e;
  if ((e = dalloc((void**)&slot_len, sizeof(int32_t) * P.nchunks, st)) != cudaSuccess) return cleanup(), e;
  if ((e = dalloc((void**)&block_sums, sizeof(int64_t) * nb, st)) != cudaSuccess) return cleanup(), e;
  if ((e = dalloc((void**)&flags, sizeof(unsigned int) * 2, st)) != cudaSuccess) return cleanup(), e;
  P.chunk_slot = (const int64_t*)out->bufs[0];
  P.maxlen = (const uint16_t*)out->bufs[1];
  const unsigned blocks = (unsigned)((P.nchunks + kWarps - 1) / kWarps);
  if (M.index_bits == 32)
    k_pack_count<int32_t><<<blocks, kThreads, 0, st>>>(M, P, slot_len, (uint16_t*)out->bufs[1]);
  else
    k_pack_count<int64_t><<<blocks, kThreads, 0, st>>>(M, P, slot_len, (uint16_t*)out->bufs[1]);
  if ((e = cudaGetLastError()) != cudaSuccess) return cleanup(), e;
  int64_t* cs = (int64_t*)out->bufs[0];
  if ((e = launch_scan_tiles(slot_len, P.nchunks, cs, cs + P.nchunks, block_sums, st)) != cudaSuccess)
    return cleanup(), e;
  int64_t slot_rows = 0;
  if ((e = cudaMemcpyAsync(&slot_rows, cs + P.nchunks, sizeof(int64_t), cudaMemcpyDeviceToHost, st)) !=
      cudaSuccess)
    return cleanup(), e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cleanup(), e;
  P.slot_rows = slot_rows;
  if ((e = dalloc(&out->bufs[4], sizeof(float) * (size_t)(P.nchunks * P.na * 32), st)) != cudaSuccess)
    return cleanup(), e;
  P.R = (const float*)out->bufs[4];
  for (int attempt = 0; attempt < 2; ++attempt) {
    const int cb = col_bytes_of(P), nb2 = cnt_bytes_of(P);
    // 16 spare elements keep every bulk prefetch inside its allocation
    if ((e = dalloc(&out->bufs[2], (size_t)(slot_rows * 32 + 16) * cb, st)) != cudaSuccess)
      return cleanup(), e;
    if (nb2 && (e = dalloc(&out->bufs[3], (size_t)(slot_rows * 32 + 16) * nb2, st)) != cudaSuccess)
      return cleanup(), e;
    P.col = out->bufs[2];
    P.cnt = out->bufs[3];
    if ((e = cudaMemsetAsync(flags, 0, sizeof(unsigned int) * 2, st)) != cudaSuccess) return cleanup(), e;
    e = dispatch_pack(P, [&](auto mode, auto* cntt) -> cudaError_t {
      using CntT = std::remove_pointer_t<decltype(cntt)>;
      constexpr int MODE = decltype(mode)::value;
      if (M.index_bits == 32)
        k_pack_fill<int32_t, MODE, CntT><<<blocks, kThreads, 0, st>>>(
            M, P, out->bufs[2], (CntT*)out->bufs[3], (float*)out->bufs[4], flags);
      else
        k_pack_fill<int64_t, MODE, CntT><<<blocks, kThreads, 0, st>>>(
            M, P, out->bufs[2], (CntT*)out->bufs[3], (float*)out->bufs[4], flags);
      return cudaGetLastError();
    });
    if (e != cudaSuccess) return cleanup(), e;
    unsigned int hf = 0;
    if ((e = cudaMemcpyAsync(&hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return cleanup(), e;
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cleanup(), e;
    if (!(hf & 1u) || P.ent_mode == ENT_I32) break;
    // a column outside the window: repack with int32 columns
    dfree(out->bufs[2], st);
    dfree(out->bufs[3], st);
    out->bufs[2] = out->bufs[3] = nullptr;
    P.ent_mode = ENT_I32;
  }
  cleanup();
  for (void* b : out->bufs)  // the L2 bulk prefetch needs 16-byte aligned ranges
    if (reinterpret_cast<uintptr_t>(b) & 15u) return cudaErrorMisalignedAddress;
  out->bytes = pack_sweep_bytes(P) - P.ns * 12;
  return cudaSuccess;
}

cudaError_t launch_vi_chunks(const ViPack& P, int64_t c_begin, int64_t c_end, const float* Vin,
                             float* Vout, int32_t* pi, unsigned long long* resid, cudaStream_t st,
                             int tune, unsigned int* err) {
  if (c_end <= c_begin) return cudaSuccess;
  if ((tune & VI_TUNE_TMA) && P.ent_mode == ENT_PACKED && err && P.na <= 32) {
    // staging shape: chunks per super-chunk, stages, entry bytes per stage
    auto run = [&](auto kern, int sc_chunks, int bytes) -> cudaError_t {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
      if (e != cudaSuccess) return e;
      int per_sm = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, bytes);
      if (e != cudaSuccess) return e;
      const int64_t n_sc = (c_end - c_begin + sc_chunks - 1) / sc_chunks;
      const int64_t cap = (int64_t)std::max(per_sm, 1) * sm_count_pack();
      const unsigned grid = (unsigned)std::min(n_sc, cap);
      kern<<<grid, kThreads, bytes, st>>>(P, (int)c_begin, (int)c_end, Vin, Vout, pi, resid, err);
      return cudaGetLastError();
    };
    // measured on c2: 2 chunks x 2 stages 2.0 TB/s; 4 stages (1 CTA/SM) 1.0,
    // 4 chunks x 3 stages 1.4, 1 chunk x 4 stages 1.3; the register-streaming
    // lean sweep 3.9: with 8-16 resident warps the V-gather chains, not DRAM
    // latency, bound the staged sweep
    return run(k_vi_tma<2, 2, 40 * 1024>, 2, 2 * sc_stage_bytes<2, 40 * 1024>(P.na, P.na_pad));
  }
  const int prefetch = tune & (PF_NEXT | PF_CURRENT);
  return dispatch_pack(P, [&](auto mode, auto* cntt) -> cudaError_t {
    using CntT = std::remove_pointer_t<decltype(cntt)>;
    constexpr int MODE = decltype(mode)::value;
    const bool lean = MODE == ENT_PACKED && (tune & VI_TUNE_LEAN);
    auto kern = lean ? k_vi_chunks<MODE, CntT, (MODE == ENT_PACKED ? 2 : 0)> : k_vi_chunks<MODE, CntT, 0>;
    const int64_t need = (c_end - c_begin + kWarps - 1) / kWarps;
    const int64_t cap = (int64_t)occupancy((const void*)kern) * sm_count_pack();
    const unsigned grid = (unsigned)std::min(need, cap);
    kern<<<grid, kThreads, 0, st>>>(P, (int)c_begin, (int)c_end, Vin, Vout, pi, resid, prefetch);
    return cudaGetLastError();
  });
}

cudaError_t launch_vi_layered(const ViPack& P, float* V, int32_t* pi, unsigned int* sync, int groups,
                              cudaStream_t st, int tune) {
  const int prefetch = tune & (PF_NEXT | PF_CURRENT);
  return dispatch_pack(P, [&](auto mode, auto* cntt) -> cudaError_t {
    using CntT = std::remove_pointer_t<decltype(cntt)>;
    constexpr int MODE = decltype(mode)::value;
    const bool lean = MODE == ENT_PACKED && (tune & VI_TUNE_LEAN);
    auto kern = lean ? k_vi_layered<MODE, CntT, (MODE == ENT_PACKED ? 2 : 0)> : k_vi_layered<MODE, CntT, 0>;
    const int64_t cap = (int64_t)occupancy((const void*)kern) * sm_count_pack();
    int G = groups;
    if (G <= 0) {
      // enough warps for one layer's chunks: split actions while that adds warps
      G = 1;
      while (G < 8 && G * 2 <= P.na && P.cpl * G * 2 <= cap * kWarps) G *= 2;
    }
    if (G != 1 && G != 2 && G != 4 && G != 8) return cudaErrorInvalidValue;
    const int cpc = kWarps / G;
    const int64_t need = (P.cpl + cpc - 1) / cpc;
    int grid = (int)std::min(need, cap);
    if (grid < 1) grid = 1;
    ViPack Pc = P;
    int pf = prefetch;
    WaitBound wb = wait_bound_from_env();
    void* args[] = {(void*)&Pc, (void*)&G, (void*)&V, (void*)&pi, (void*)&sync, (void*)&pf, (void*)&wb};
    return cudaLaunchCooperativeKernel((const void*)kern, dim3((unsigned)grid), dim3(kThreads), args, 0, st);
  });
}

size_t vi_batch_table_bytes(int job_cap, int layer_cap) {
  return kViBatchJobsOffset + sizeof(ViJob) * (size_t)job_cap + sizeof(int) * (size_t)(job_cap + 1) +
         sizeof(int) * (size_t)layer_cap;
}

namespace {
struct PackKey {
  int ent_mode, count_type;
};
template <typename F>
cudaError_t dispatch_key(const PackKey& k, F&& f) {
  ViPack P{};
  P.ent_mode = k.ent_mode;
  P.count_type = k.count_type;
  return dispatch_pack(P, f);
}
}  // namespace

int vi_batch_capacity(int ent_mode, int count_type, int tune) {
  int cap = 0;
  dispatch_key(PackKey{ent_mode, count_type}, [&](auto mode, auto* cntt) -> cudaError_t {
    using CntT = std::remove_pointer_t<decltype(cntt)>;
    constexpr int MODE = decltype(mode)::value;
    const bool lean = MODE == ENT_PACKED && (tune & VI_TUNE_LEAN);
    auto kern = lean ? k_vi_batch<MODE, CntT, (MODE == ENT_PACKED ? 2 : 0)> : k_vi_batch<MODE, CntT, 0>;
    cap = occupancy((const void*)kern) * sm_count_pack();
    return cudaSuccess;
  });
  return cap;
}

cudaError_t launch_vi_batch(const void* table, int job_cap, int layer_cap, int ent_mode, int count_type,
                            int groups, int grid, int tune, int* done, unsigned int* err, cudaStream_t st) {
  if (groups != 1 && groups != 2 && groups != 4 && groups != 8) return cudaErrorInvalidValue;
  if (job_cap > kViBatchJobCap) return cudaErrorInvalidValue;  // the kernel's shared prefix sums
  const int prefetch = tune & (PF_NEXT | PF_CURRENT);
  return dispatch_key(PackKey{ent_mode, count_type}, [&](auto mode, auto* cntt) -> cudaError_t {
    using CntT = std::remove_pointer_t<decltype(cntt)>;
    constexpr int MODE = decltype(mode)::value;
    const bool lean = MODE == ENT_PACKED && (tune & VI_TUNE_LEAN);
    auto kern = lean ? k_vi_batch<MODE, CntT, (MODE == ENT_PACKED ? 2 : 0)> : k_vi_batch<MODE, CntT, 0>;
    const int cap = occupancy((const void*)kern) * sm_count_pack();
    if (grid < 1 || grid > cap) return cudaErrorInvalidValue;  // CTAs must be co-resident
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const unsigned char* tb = reinterpret_cast<const unsigned char*>(table);
    int pf = prefetch;
    const WaitBound wb = wait_bound_from_env();
    return cudaLaunchKernelEx(&cfg, kern, tb, job_cap, groups, done, layer_cap, err, pf, wb);
  });
}

}  // namespace e2e
