// K5 + K6: the sliced copy of a model that value iteration streams, and the
// sweeps over it.
//
// Layout: row-sorted groups.  States are taken in groups of G = max(1, 256/na)
// consecutive states of one layer (a group never crosses a layer boundary;
// the last group of a layer may be partial), i.e. at most 256 rows (s, a).
// Within a group the rows are ordered by length, longest first (stable in row
// order; lengths above 63 count as 63), and cut into slices of 32: lane l of
// slice j holds the row at sorted position 32j + l.  Slice j stores
// maxlen[group][j] slot rows of 32 entries, so entry k of the slice's 32 rows
// is one coalesced line:
//   slot (chunk_slot[group] + sum_{i<j} maxlen[group][i] + k) * 32 + l.
// Rows shorter than their slice's maxlen are padded with count 0.  Sorting
// keeps rows of similar length in a slice: on the 200x200x120 model the
// padding is 7 % of the entries (33.7 % with one row per lane for 32 states of
// one action).  Per sorted position the group stores the row (perm, one byte:
// s_local * na + a) and its R.
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
// operands).  A padding slot therefore points at the row's own cell in layer
// t+1, whose value is final before layer t is computed in any schedule, never
// at memory the current sweep has not written yet.  The rows' Q values go to
// shared memory at (s_local, a); the first-maximum argmax then runs per state
// in action order (the reference's select_best_action, src/spvi_2.cu:93-122:
// start -1e6 / -1, strict '>', NaN never taken).  Values are bit-identical to
// the CSR sweep.
//
// Per row the sweep reads (offset + count) per padded entry, R, one perm byte
// and the gathered V; there is no row pointer.
#include <math.h>

#include <algorithm>
#include <cstdlib>
#include <type_traits>

#include "internal.h"

namespace e2e {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kSlices = 8;          // slices of 32 rows per group
constexpr int kGroupRows = 256;     // rows per group (G * na <= 256)
constexpr int kQStride = 512;       // shared Q floats per group: G * (na + 1) <= 512, plus a spare
constexpr int kLenKeys = 64;        // sort keys: row lengths 0..63, longer rows as 63
constexpr int PF_NEXT = VI_TUNE_PF_NEXT;
constexpr int PF_CURRENT = VI_TUNE_PF_CURRENT;
constexpr long long kBarrierSpinLimit = 1ll << 22;
constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s
constexpr unsigned kFull = 0xffffffffu;

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

// Position of group c: first state, layer, its index in the layer, states and rows.
struct GroupPos {
  int64_t s0;
  int t, sl0, gvalid, rows;
};

// group indices, layer sizes and grid sides fit in 32 bits (checked on the host)
__device__ __forceinline__ GroupPos group_pos(const ViPack& P, int c) {
  GroupPos r;
  const int cpl = (int)P.cpl, nc = (int)P.nc;
  r.t = c / cpl;
  r.sl0 = (c - r.t * cpl) * P.gs;
  r.gvalid = min(P.gs, nc - r.sl0);
  r.s0 = (int64_t)r.t * nc + r.sl0;
  r.rows = r.gvalid * P.na;
  return r;
}

// Window base of the columns of state s (window-offset layouts):
// (t+1) g^2 + (i-del) g + (j-del) = s + g^2 - del (g+1) for s = t g^2 + i g + j.
// Only states that own rows (s < n_row_states, t+1 < nlayers) have entries.
__device__ __forceinline__ int64_t window_base(const ViPack& P, int64_t s) {
  if (s >= P.n_row_states) return 0;
  return s + P.nc - P.delg;
}

// the row (s_local, a) at a sorted position from its perm byte
__device__ __forceinline__ void row_of(const ViPack& P, int p, int& s_local, int& a) {
  if (P.na_shift >= 0) {
    s_local = p >> P.na_shift;
    a = p & (P.na - 1);
  } else {
    s_local = p / P.na;
    a = p - s_local * P.na;
  }
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
  // entries k0 .. k0+n-1 (n <= B) of this lane's row, zeros beyond
  template <int B>
  __device__ __forceinline__ void load(int k0, int n, ColT (&o)[B], CntT (&w)[B]) const {
    const ColT* cp = col + (int64_t)k0 * 32;
    const CntT* wp = MODE != ENT_PACKED ? cnt + (int64_t)k0 * 32 : nullptr;
    if (n == B) {
#pragma unroll
      for (int j = 0; j < B; ++j) {
        o[j] = ld_stream(cp + j * 32);
        w[j] = MODE != ENT_PACKED ? ld_stream(wp + j * 32) : (CntT)0;
      }
      return;
    }
#pragma unroll
    for (int j = 0; j < B; ++j) {
      o[j] = 0;
      w[j] = 0;
      if (j < n) {
        o[j] = ld_stream(cp + j * 32);
        if (MODE != ENT_PACKED) w[j] = ld_stream(wp + j * 32);
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

// Q of the rows of this warp's slices of group c (slices j0, j0 + jstep, ...)
// into q[s_local * (na + 1) + a]: the row's FMA chain in entry order, then
// finish_row with R = rfun(sorted position, s_local, a).  Entries come B at a
// time without branches: positions at or beyond the slice's maxlen reload
// the slice's last entry of the row (an L1 hit) with weight 0, and
// fma(0, v, acc) == acc for the finite v it points at.
template <int MODE, typename CntT, bool COHERENT, int B, typename RF>
__device__ __forceinline__ void group_q(const ViPack& P, int c, const GroupPos& gp, int lane, int j0,
                                        int jstep, const float* Vin, float* q, RF&& rfun) {
  using ColT = typename Entries<MODE, CntT>::ColT;
  const int nsl = (gp.rows + 31) >> 5;
  // slot rows of the slices (lane j: slice j) and their inclusive prefix
  const int mlj = lane < kSlices ? (int)__ldg(P.maxlen + (int64_t)c * kSlices + lane) : 0;
  int incl = mlj;
#pragma unroll
  for (int o = 1; o < kSlices; o <<= 1) {
    const int t2 = __shfl_up_sync(kFull, incl, o);
    if (lane >= o) incl += t2;
  }
  // everything the slice loop needs, in registers
  const int64_t e0 = __ldg(P.chunk_slot + c) * 32 + lane;
  const ColT* colg = reinterpret_cast<const ColT*>(P.col) + e0;
  const CntT* cntg = MODE == ENT_PACKED ? nullptr : reinterpret_cast<const CntT*>(P.cnt) + e0;
  const uint8_t* permg = P.perm + (int64_t)c * kGroupRows + lane;
  const int na = P.na, na1 = na + 1, na_shift = P.na_shift;
  const int64_t nrs = P.n_row_states, woff = P.nc - P.delg;
  const bool counts = P.count_type != VAL_F32;
  const float fn = (float)P.nrzns;
  for (int j = j0; j < nsl; j += jstep) {
    const int ml = __shfl_sync(kFull, mlj, j);
    const int pre = __shfl_sync(kFull, incl, j) - ml;
    const int pos = (j << 5) + lane;
    // unused lanes of a partial group's last slice read the padding the pack
    // holds for them (perm 0, count 0, R 0) and write a spare slot of q
    const bool used = pos < gp.rows;
    const int p = __ldg(permg + (j << 5));
    int s_local, a;
    if (na_shift >= 0) {
      s_local = p >> na_shift;
      a = p & (na - 1);
    } else {
      s_local = p / na;
      a = p - s_local * na;
    }
    const int64_t s = gp.s0 + s_local;
    // window base of the row's columns: s + g^2 - del (g+1) (rows exist only for s < n_row_states)
    const float* vb = MODE == ENT_I32 ? Vin : Vin + (s < nrs ? s + woff : 0);
    const ColT* ce = colg + (pre << 5);
    const CntT* cw = MODE == ENT_PACKED ? nullptr : cntg + (pre << 5);
    const float r = rfun(pos, s_local, a);
    float acc = 0.f;
    for (int k0 = 0; k0 < ml; k0 += B) {
      ColT o[B];
      CntT w[B];
#pragma unroll
      for (int jj = 0; jj < B; ++jj) {
        const int k = min(k0 + jj, ml - 1);
        o[jj] = ld_stream(ce + (k << 5));
        w[jj] = MODE != ENT_PACKED ? ld_stream(cw + (k << 5)) : (CntT)0;
      }
      float v[B], f[B];
#pragma unroll
      for (int jj = 0; jj < B; ++jj) {
        uint32_t idx;
        decode<MODE, ColT, CntT>(o[jj], w[jj], idx, f[jj]);
        if (k0 + jj >= ml) f[jj] = 0.f;
        v[jj] = ld_value<COHERENT>(vb + idx);
      }
#pragma unroll
      for (int jj = 0; jj < B; ++jj) acc = fmaf(f[jj], v[jj], acc);
    }
    q[used ? s_local * na1 + a : kQStride] = counts ? r + acc / fn : r + acc;  // finish_row
  }
}

// First maximum over actions [a0, a1) of state s_local of a group, from q
// (strict '>', NaN never taken: bq stays -inf / ba INT_MAX without a candidate).
__device__ __forceinline__ void state_best(const ViPack& P, const float* q, int s_local, int a0, int a1,
                                           float& bq, int& ba) {
  const int na1 = P.na + 1;
  bq = -INFINITY;
  ba = 0x7fffffff;
  for (int a = a0; a < a1; ++a) {
    const float qa = q[s_local * na1 + a];
    if (!isnan(qa) && qa > bq) {
      bq = qa;
      ba = a;
    }
  }
}

// The first maximum of every state of the group, then out(s_local, bq, ba).
// With lps > 1 lanes per state, each lane scans a block of apl actions and the
// blocks meet by shuffles: a later block wins only with a larger value, an
// equal value keeps the lower action -- the sequential first maximum.
template <typename OUT>
__device__ __forceinline__ void group_argmax(const ViPack& P, const GroupPos& gp, int lane, const float* q,
                                             OUT&& out) {
  const int lps = P.lps;
  if (lps > 1) {
    const int sl = lane >> (__ffs(lps) - 1), part = lane & (lps - 1);
    const int a0 = min(P.na, part * P.apl), a1 = min(P.na, a0 + P.apl);
    float bq = -INFINITY;
    int ba = 0x7fffffff;
    if (sl < gp.gvalid) state_best(P, q, sl, a0, a1, bq, ba);
    for (int o = lps >> 1; o > 0; o >>= 1) {
      const float oq = __shfl_xor_sync(kFull, bq, o);
      const int oa = __shfl_xor_sync(kFull, ba, o);
      if (oq > bq || (oq == bq && oa < ba)) {
        bq = oq;
        ba = oa;
      }
    }
    if (part == 0 && sl < gp.gvalid) out(sl, bq, ba);
  } else {
    for (int sl = lane; sl < gp.gvalid; sl += 32) {
      float bq;
      int ba;
      state_best(P, q, sl, 0, P.na, bq, ba);
      out(sl, bq, ba);
    }
  }
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

template <int MODE, typename CntT>
struct Widths {
  static constexpr int col = MODE == ENT_OFF16 ? 2 : 4;
  static constexpr int cnt = MODE == ENT_PACKED ? 0 : (int)sizeof(CntT);
};

// L2 prefetch of group c: entry streams, R and perm (bulk prefetch, one lane)
__device__ __forceinline__ void prefetch_group(const ViPack& P, int c, int col_bytes, int cnt_bytes) {
  const int64_t s0 = __ldg(P.chunk_slot + c), s1 = __ldg(P.chunk_slot + c + 1);
  const int64_t n = (s1 - s0) * 32;
  if (n > 0) {
    prefetch_l2(reinterpret_cast<const char*>(P.col) + s0 * 32 * col_bytes, (uint32_t)(n * col_bytes));
    if (cnt_bytes)
      prefetch_l2(reinterpret_cast<const char*>(P.cnt) + s0 * 32 * cnt_bytes, (uint32_t)(n * cnt_bytes));
  }
  prefetch_l2(P.R + (int64_t)c * kGroupRows, (uint32_t)(kGroupRows * 4));
  prefetch_l2(P.perm + (int64_t)c * kGroupRows, (uint32_t)kGroupRows);
}

// VAR 0: 8 entries a batch, 5 CTAs per SM; VAR 1: 4 entries, 8 CTAs per SM
// (latency hidden by more resident warps instead)
template <int MODE, int VAR>
struct MinBlocks {
  static constexpr int value = MODE != ENT_PACKED ? 3 : (VAR == 0 ? 5 : 8);
};
template <int VAR>
struct Batch {
  static constexpr int value = VAR == 0 ? 8 : 4;
};

// One Jacobi sweep over groups [c_begin, c_end): warp per group, grid-stride;
// prefetch bits: PF_NEXT = the warp's next group, PF_CURRENT = the group it starts.
template <int MODE, typename CntT, int VAR>
__global__ void __launch_bounds__(kThreads, MinBlocks<MODE, VAR>::value)
    k_vi_chunks(ViPack P, int c_begin, int c_end, const float* __restrict__ Vin, float* Vout, int32_t* pi,
                unsigned long long* resid, int prefetch) {
  __shared__ float qs[kWarps][kQStride + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = gridDim.x * kWarps;
  float* q = qs[wid];
  double dmax = 0.0;
  for (int c = c_begin + blockIdx.x * kWarps + wid; c < c_end; c += nw) {
    if ((prefetch & PF_NEXT) && lane == 0 && c + nw < c_end)
      prefetch_group(P, c + nw, Widths<MODE, CntT>::col, Widths<MODE, CntT>::cnt);
    if ((prefetch & PF_CURRENT) && lane == 0) prefetch_group(P, c, Widths<MODE, CntT>::col, Widths<MODE, CntT>::cnt);
    const GroupPos gp = group_pos(P, c);
    const float* Rg = P.R + (int64_t)c * kGroupRows;
    group_q<MODE, CntT, false, Batch<VAR>::value>(P, c, gp, lane, 0, 1, Vin, q,
                                                  [&](int pos, int, int) { return ld_stream(Rg + pos); });
    __syncwarp();
    group_argmax(P, gp, lane, q, [&](int sl, float bq, int ba) {
      float vout;
      int32_t pout;
      finish_state(bq, ba, vout, pout);
      const int64_t s = gp.s0 + sl;
      if (resid) dmax = fmax(dmax, fabs((double)vout - (double)Vin[s]));
      Vout[s] = vout;
      pi[s] = pout;
    });
    __syncwarp();  // q is rewritten by the next group
  }
  if (resid) {
    for (int off = 16; off > 0; off >>= 1) dmax = fmax(dmax, __shfl_xor_sync(kFull, dmax, off));
    __shared__ double wmax[kWarps];
    if (lane == 0) wmax[wid] = dmax;
    __syncthreads();
    if (threadIdx.x == 0) {
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
// share a group of states, each taking every groups-th slice; their rows' Q
// meet in shared memory and the first warp takes the argmax.  With PF_NEXT,
// each group's data for the next layer is prefetched into L2 before this
// layer's work, so HBM streams layer t-1 while layer t computes.
template <int MODE, typename CntT, int VAR>
__global__ void __launch_bounds__(kThreads, MinBlocks<MODE, VAR>::value)
    k_vi_layered(ViPack P, int groups, float* V, int32_t* pi, unsigned int* sync, int prefetch, WaitBound wb) {
  __shared__ float qs[kWarps][kQStride + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int cpc = kWarps / groups;  // groups of states per CTA iteration
  const int grp = wid % groups, slot_in_cta = wid / groups;
  float* q = qs[slot_in_cta];
  const int cpl = (int)P.cpl;
  unsigned int gen = 0;
  for (int t = P.nlayers - 1; t >= 0; --t) {
    for (int b = blockIdx.x * cpc; b < cpl; b += gridDim.x * cpc) {
      const int cc = b + slot_in_cta;
      const bool active = cc < cpl;
      const int c = t * cpl + cc;
      GroupPos gp{0, 0, 0, 0, 0};
      if (active) {
        if ((prefetch & PF_NEXT) && lane == 0 && grp == 0 && t > 0)
          prefetch_group(P, c - cpl, Widths<MODE, CntT>::col, Widths<MODE, CntT>::cnt);
        gp = group_pos(P, c);
        const float* Rg = P.R + (int64_t)c * kGroupRows;
        group_q<MODE, CntT, true, Batch<VAR>::value>(P, c, gp, lane, grp, groups, V, q,
                                                     [&](int pos, int, int) { return ld_stream(Rg + pos); });
      }
      if (groups > 1) __syncthreads();
      else __syncwarp();
      if (active && grp == 0) {
        group_argmax(P, gp, lane, q, [&](int sl, float bq, int ba) {
          float vout;
          int32_t pout;
          finish_state(bq, ba, vout, pout);
          V[gp.s0 + sl] = vout;
          pi[gp.s0 + sl] = pout;
        });
      }
      if (groups > 1) __syncthreads();
      else __syncwarp();
    }
    if (t > 0) {
      ++gen;
      if (!grid_barrier(sync, gen * gridDim.x, wb)) return;
    }
  }
}

// Many layered solves in one persistent launch.  Step k covers layer
// nlayers-1-k of every job that has more than k layers (jobs sorted by layer
// count, so those are a prefix and their groups a contiguous item range).
// There is no grid-wide barrier: a group of layer t waits only until its own
// job's layer t+1 is complete (done[job][t+1] == groups per layer), and each
// finished group adds one to done[job][t].  Every CTA takes its items in step
// order and all CTAs are resident (cooperative launch), so each wait is for
// items of an earlier step that are finished or running; the waits are
// bounded and a timeout sets bit 2 of err and lets the rest drain quickly.
// Jobs with a target take R of the cells around it from their Rwin table,
// and the target's own cells are terminal: the reference leaves such a
// sample in place with reward 0 (src/build_model.cu:523-545), i.e. one entry
// (the cell at t+1, count nrzns) and R = 0, evaluated here with the same
// operations as that row.
template <int MODE, int VAR>
struct BatchMinBlocks {  // the job lookup needs a few more registers than k_vi_layered
  static constexpr int value = MODE != ENT_PACKED ? 3 : (VAR == 0 ? 4 : 5);
};

template <int MODE, typename CntT, int VAR>
__global__ void __launch_bounds__(kThreads, BatchMinBlocks<MODE, VAR>::value)
    k_vi_batch(const unsigned char* table, int job_cap, int groups, int* done, int layer_cap,
               unsigned int* err, int prefetch, WaitBound wb) {
  __shared__ float qs[kWarps][kQStride + 1];
  const ViBatchHeader* H = reinterpret_cast<const ViBatchHeader*>(table);
  const ViJob* jobs = reinterpret_cast<const ViJob*>(table + kViBatchJobsOffset);
  const int* cum = reinterpret_cast<const int*>(jobs + job_cap);
  const int* nact = cum + job_cap + 1;
  const int L = H->max_layers;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int cpc = kWarps / groups;
  const int grp = wid % groups, slot_in_cta = wid / groups;
  float* q = qs[slot_in_cta];
  for (int k = 0; k < L; ++k) {
    const int nj = nact[k];
    const int n_items = cum[nj];
    for (int b = blockIdx.x * cpc; b < n_items; b += gridDim.x * cpc) {
      const int item = b + slot_in_cta;
      const bool active = item < n_items;
      int jid = 0, c = 0, t = 0;
      int* done_slot = nullptr;
      bool skip = false;
      GroupPos gp{0, 0, 0, 0, 0};
      if (active) {
        int lo = 0, hi = nj - 1;  // last job with cum[job] <= item
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (__ldg(cum + mid) <= item) lo = mid;
          else hi = mid - 1;
        }
        jid = lo;
        const ViJob& J = jobs[jid];
        const ViPack& P = J.P;
        const int cpl = (int)P.cpl;
        t = P.nlayers - 1 - k;
        c = t * cpl + (item - __ldg(cum + jid));
        done_slot = done + (int64_t)jid * layer_cap + t;
        if ((prefetch & PF_NEXT) && lane == 0 && grp == 0 && t > 0)
          prefetch_group(P, c - cpl, Widths<MODE, CntT>::col, Widths<MODE, CntT>::cnt);
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
          ok = __shfl_sync(kFull, ok, 0);
          (void)ld_acquire_s32(dep);  // every lane orders its reads after the producers' writes
          skip = !ok;                 // give up this group: nothing computed, nothing written
        }
        gp = group_pos(P, c);
        if (!skip) {
          const float* Rg = P.R + (int64_t)c * kGroupRows;
          const bool win = J.Rwin && t + 1 < P.nlayers;
          const int na = P.na;
          group_q<MODE, CntT, true, Batch<VAR>::value>(
              P, c, gp, lane, grp, groups, J.V, q, [&](int pos, int s_local, int a) {
                const int sl = gp.sl0 + s_local;
                if (win && sl >= J.wi0 * P.g && sl < (J.wi0 + J.wh) * P.g) {
                  const int i = sl / P.g, jj = sl - i * P.g;
                  const int wi = i - J.wi0, wj = jj - J.wj0;
                  if (wj >= 0 && wj < J.ww)
                    return ld_stream(J.Rwin + (((int64_t)t * J.wh + wi) * J.ww + wj) * na + a);
                }
                return ld_stream(Rg + pos);
              });
        }
      }
      if (groups > 1) __syncthreads();
      else __syncwarp();
      if (active && grp == 0) {
        const ViJob& J = jobs[jid];
        const ViPack& P = J.P;
        if (!skip) {
          const int nc = (int)P.nc;
          group_argmax(P, gp, lane, q, [&](int sl, float bq, int ba) {
            const int64_t s = gp.s0 + sl;
            if (J.Rwin && t + 1 < P.nlayers) {
              const int cl = gp.sl0 + sl;
              const int i = cl / P.g, j = cl - (cl / P.g) * P.g;
              if (i >= J.ti && i < J.ti + J.tsg && j >= J.tj && j < J.tj + J.tsg) {
                const float v = ld_value<true>(J.V + s + nc);  // the same cell, layer t+1
                const float acc = fmaf((float)P.nrzns, v, 0.f);
                const float qt = finish_row(0.f, acc, 0.f, P.nrzns, true);
                bq = -INFINITY;
                ba = 0x7fffffff;
                if (!isnan(qt)) {
                  bq = qt;
                  ba = 0;
                }
              }
            }
            float vout;
            int32_t po;
            finish_state(bq, ba, vout, po);
            J.V[s] = vout;
            J.pi[s] = po;
          });
        }
        __syncwarp();
        if (lane == 0) {
          __threadfence();  // this group's values before its completion count
          atomicAdd(done_slot, 1);
        }
      }
      if (groups > 1) __syncthreads();
      else __syncwarp();
    }
  }
}

// ---- pack construction ------------------------------------------------------------

// Per group (warp per group): the rows' lengths, their order (longest first,
// stable; a counting sort on min(len, 63)), perm and R in that order, the
// slices' maxlen and their sum.
template <typename PtrT>
__global__ void __launch_bounds__(kThreads) k_pack_count(ViModel M, ViPack P, int32_t* slot_len,
                                                         uint16_t* maxlen, uint8_t* perm, float* Rs) {
  __shared__ int lens[kWarps][kGroupRows];
  __shared__ int slen[kWarps][kGroupRows];
  __shared__ int off[kWarps][kLenKeys];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int c = blockIdx.x * kWarps + wid;
  if (c >= P.nchunks) return;  // warp-level work only: no block barrier below
  const GroupPos gp = group_pos(P, c);
  const PtrT* rp = reinterpret_cast<const PtrT*>(M.row_ptr);
  const int na = P.na;
  for (int r = lane; r < kGroupRows; r += 32) {
    int len = 0;
    if (r < gp.rows) {
      const int64_t s = gp.s0 + r / na;
      if (s < P.n_row_states) {
        const int64_t row = s * na + (r % na);
        len = (int)((int64_t)rp[row + 1] - (int64_t)rp[row]);
      }
    }
    lens[wid][r] = len;
  }
  for (int k = lane; k < kLenKeys; k += 32) off[wid][k] = 0;
  __syncwarp();
  // key 0 = longest rows
  auto key_of = [](int len) { return kLenKeys - 1 - min(len, kLenKeys - 1); };
  for (int r = lane; r < gp.rows; r += 32) atomicAdd(&off[wid][key_of(lens[wid][r])], 1);
  __syncwarp();
  {  // exclusive prefix of the key counts, two keys a lane
    const int v0 = off[wid][2 * lane], v1 = off[wid][2 * lane + 1];
    int incl = v0 + v1;
    for (int o = 1; o < 32; o <<= 1) {
      const int t2 = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t2;
    }
    const int ex = incl - v0 - v1;
    __syncwarp();
    off[wid][2 * lane] = ex;
    off[wid][2 * lane + 1] = ex + v0;
  }
  __syncwarp();
  // stable placement, 32 rows at a time, rows of equal length in
  // action-major order (u = a * gvalid + s_local): a slice then holds few
  // actions over consecutive states, whose V gathers share cache lines
  for (int base = 0; base < gp.rows; base += 32) {
    const int u = base + lane;
    const bool has = u < gp.rows;
    const int ua = has ? u / gp.gvalid : 0;
    const int r = has ? (u - ua * gp.gvalid) * na + ua : 0;
    const int key = has ? key_of(lens[wid][r]) : kLenKeys + lane;
    const unsigned m = __match_any_sync(kFull, key);
    const int rank = __popc(m & ((1u << lane) - 1u));
    const int pos = has ? off[wid][key] + rank : 0;
    __syncwarp();
    if (has && rank == 0) off[wid][key] += __popc(m);
    __syncwarp();
    if (has) {
      perm[(int64_t)c * kGroupRows + pos] = (uint8_t)r;
      slen[wid][pos] = lens[wid][r];
      Rs[(int64_t)c * kGroupRows + pos] = M.R[(gp.s0 + r / na) * na + (r % na)];
    }
  }
  __syncwarp();
  for (int pos = gp.rows + lane; pos < kGroupRows; pos += 32) {
    perm[(int64_t)c * kGroupRows + pos] = 0;
    Rs[(int64_t)c * kGroupRows + pos] = 0.f;
  }
  int total = 0;
  for (int j = 0; j < kSlices; ++j) {
    const int pos = (j << 5) + lane;
    const unsigned ml = __reduce_max_sync(kFull, pos < gp.rows ? (unsigned)slen[wid][pos] : 0u);
    if (lane == 0) maxlen[(int64_t)c * kSlices + j] = (uint16_t)ml;
    total += (int)ml;
  }
  if (lane == 0) slot_len[c] = total;
}

// scatter the CSR rows into the group layout; flags[0] |= 1 when a window
// offset does not fit 16 bits (the caller then packs with int32 columns)
template <typename PtrT, int MODE, typename CntT>
__global__ void __launch_bounds__(kThreads) k_pack_fill(ViModel M, ViPack P, void* colv, CntT* cnt,
                                                        unsigned int* flags) {
  const int lane = threadIdx.x & 31;
  const int c = blockIdx.x * kWarps + (threadIdx.x >> 5);
  if (c >= P.nchunks) return;
  const GroupPos gp = group_pos(P, c);
  const PtrT* rp = reinterpret_cast<const PtrT*>(M.row_ptr);
  const CntT* src = reinterpret_cast<const CntT*>(M.cnt);
  const int na = P.na;
  int64_t slot = P.chunk_slot[c];
  bool bad = false;
  for (int j = 0; j < kSlices; ++j) {
    const int ml = P.maxlen[(int64_t)c * kSlices + j];
    const int pos = (j << 5) + lane;
    const bool valid = pos < gp.rows;
    const int r = valid ? P.perm[(int64_t)c * kGroupRows + pos] : 0;
    int s_local, a;
    row_of(P, r, s_local, a);
    const int64_t s = gp.s0 + s_local;
    const bool has = valid && s < P.n_row_states;
    int64_t rs = 0, len = 0;
    if (has) {
      const int64_t row = s * na + a;
      rs = (int64_t)rp[row];
      len = (int64_t)rp[row + 1] - rs;
    }
    const int64_t base = MODE == ENT_I32 ? 0 : window_base(P, s);
    // padding (count 0) points at the row's own cell in layer t+1, finished
    // before layer t in every schedule, so the gathered value is finite and
    // fma(0, v, acc) leaves acc unchanged; unused lanes get the same index
    const int32_t pad_col = (int32_t)(gp.t + 1 < P.nlayers ? s + P.nc : s);
    for (int k = 0; k < ml; ++k) {
      const int64_t e = (slot + k) * 32 + lane;
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
        int64_t o = (int64_t)col - base;
        if (o < 0 || o > 65535) {
          if (valid) bad = true;
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
  // entries (with padding) + R + perm + group tables + V read + V' and policy written
  return P.slot_rows * 32 * (col_bytes_of(P) + cnt_bytes_of(P)) + P.nchunks * kGroupRows * (4 + 1) +
         P.nchunks * (8 + kSlices * 2) + P.ns * 12;
}

cudaError_t build_pack(const ViModel& M, int64_t nc, int g, int del, PackStore* out, cudaStream_t st) {
  *out = PackStore{};
  ViPack& P = out->v;
  P.ns = M.ns;
  P.nc = (nc > 0 && M.ns % nc == 0) ? nc : M.ns;
  P.nlayers = (int)(M.ns / P.nc);
  P.na = M.na;
  if (P.na < 1 || P.na > kGroupRows) return cudaErrorInvalidValue;
  P.gs = std::max(1, kGroupRows / P.na);
  P.cpl = (P.nc + P.gs - 1) / P.gs;
  P.nchunks = P.cpl * P.nlayers;
  if (P.nc >= ((int64_t)1 << 31) - 64 || P.nchunks >= ((int64_t)1 << 31) - 1)
    return cudaErrorInvalidValue;  // 32-bit group arithmetic
  P.n_row_states = M.n_row_states;
  P.na_pad = (M.na + 7) & ~7;
  P.nrzns = M.nrzns;
  P.count_type = M.count_type;
  P.g = g;
  P.del = del;
  P.delg = (int64_t)del * (g + 1);
  P.na_shift = -1;
  for (int k = 0; k < 9; ++k)
    if (P.na == (1 << k)) P.na_shift = k;
  P.lps = 1;
  while (P.lps * 2 * P.gs <= 32) P.lps *= 2;
  P.apl = (P.na + P.lps - 1) / P.lps;
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
  if ((e = dalloc(&out->bufs[1], sizeof(uint16_t) * P.nchunks * kSlices, st)) != cudaSuccess) return e;
  if ((e = dalloc(&out->bufs[4], sizeof(float) * (size_t)(P.nchunks * kGroupRows), st)) != cudaSuccess) return e;
  if ((e = dalloc(&out->bufs[5], (size_t)(P.nchunks * kGroupRows), st)) != cudaSuccess) return e;
  if ((e = dalloc((void**)&slot_len, sizeof(int32_t) * P.nchunks, st)) != cudaSuccess) return cleanup(), e;
  if ((e = dalloc((void**)&block_sums, sizeof(int64_t) * nb, st)) != cudaSuccess) return cleanup(), e;
  if ((e = dalloc((void**)&flags, sizeof(unsigned int) * 2, st)) != cudaSuccess) return cleanup(), e;
  P.chunk_slot = (const int64_t*)out->bufs[0];
  P.maxlen = (const uint16_t*)out->bufs[1];
  P.R = (const float*)out->bufs[4];
  P.perm = (const uint8_t*)out->bufs[5];
  const unsigned blocks = (unsigned)((P.nchunks + kWarps - 1) / kWarps);
  if (M.index_bits == 32)
    k_pack_count<int32_t><<<blocks, kThreads, 0, st>>>(M, P, slot_len, (uint16_t*)out->bufs[1],
                                                       (uint8_t*)out->bufs[5], (float*)out->bufs[4]);
  else
    k_pack_count<int64_t><<<blocks, kThreads, 0, st>>>(M, P, slot_len, (uint16_t*)out->bufs[1],
                                                       (uint8_t*)out->bufs[5], (float*)out->bufs[4]);
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
        k_pack_fill<int32_t, MODE, CntT><<<blocks, kThreads, 0, st>>>(M, P, out->bufs[2], (CntT*)out->bufs[3],
                                                                      flags);
      else
        k_pack_fill<int64_t, MODE, CntT><<<blocks, kThreads, 0, st>>>(M, P, out->bufs[2], (CntT*)out->bufs[3],
                                                                      flags);
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
  (void)err;
  if (c_end <= c_begin) return cudaSuccess;
  const int prefetch = tune & (PF_NEXT | PF_CURRENT);
  return dispatch_pack(P, [&](auto mode, auto* cntt) -> cudaError_t {
    using CntT = std::remove_pointer_t<decltype(cntt)>;
    constexpr int MODE = decltype(mode)::value;
    const bool lean = MODE == ENT_PACKED && (tune & VI_TUNE_LEAN);
    auto kern = lean ? k_vi_chunks<MODE, CntT, (MODE == ENT_PACKED ? 1 : 0)> : k_vi_chunks<MODE, CntT, 0>;
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
  const int nsl = (int)std::min<int64_t>(kSlices, ((int64_t)P.gs * P.na + 31) / 32);
  return dispatch_pack(P, [&](auto mode, auto* cntt) -> cudaError_t {
    using CntT = std::remove_pointer_t<decltype(cntt)>;
    constexpr int MODE = decltype(mode)::value;
    const bool lean = MODE == ENT_PACKED && (tune & VI_TUNE_LEAN);
    auto kern = lean ? k_vi_layered<MODE, CntT, (MODE == ENT_PACKED ? 1 : 0)> : k_vi_layered<MODE, CntT, 0>;
    const int64_t cap = (int64_t)occupancy((const void*)kern) * sm_count_pack();
    int G = groups;
    if (G <= 0) {
      // enough warps for one layer's groups: split slices while that adds warps
      G = 1;
      while (G < 8 && G * 2 <= nsl && P.cpl * G * 2 <= cap * kWarps) G *= 2;
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
    auto kern = lean ? k_vi_batch<MODE, CntT, (MODE == ENT_PACKED ? 1 : 0)> : k_vi_batch<MODE, CntT, 0>;
    cap = occupancy((const void*)kern) * sm_count_pack();
    return cudaSuccess;
  });
  return cap;
}

cudaError_t launch_vi_batch(const void* table, int job_cap, int layer_cap, int ent_mode, int count_type,
                            int groups, int grid, int tune, int* done, unsigned int* err, cudaStream_t st) {
  if (groups != 1 && groups != 2 && groups != 4 && groups != 8) return cudaErrorInvalidValue;
  const int prefetch = tune & (PF_NEXT | PF_CURRENT);
  return dispatch_key(PackKey{ent_mode, count_type}, [&](auto mode, auto* cntt) -> cudaError_t {
    using CntT = std::remove_pointer_t<decltype(cntt)>;
    constexpr int MODE = decltype(mode)::value;
    const bool lean = MODE == ENT_PACKED && (tune & VI_TUNE_LEAN);
    auto kern = lean ? k_vi_batch<MODE, CntT, (MODE == ENT_PACKED ? 1 : 0)> : k_vi_batch<MODE, CntT, 0>;
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
