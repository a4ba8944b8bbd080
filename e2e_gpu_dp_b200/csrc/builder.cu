// K1: fused Monte-Carlo transition builder, and K2/K3: CSR assembly.
//
// Replaces, per time layer t and action a, the reference's
//   transition_calc          src/build_model.cu:483-559  (one thread per sample,
//                            float global atomics into an ncells x (m*m+1) scratch)
//   compute_mean             :563-570
//   count_kernel + thrust::reduce + thrust::exclusive_scan   :574-594, :801-831
//   reduce_kernel            :597-644  (one thread walks 441 bins per cell)
// with one kernel over all layers:
//
//  * a CTA owns 32 cells of one layer and all actions; a warp holds 32/P
//    consecutive cells x P action lanes (P = next power of two >= actions),
//    i.e. a contiguous range of model rows.  Which cell groups a CTA takes is
//    chosen by group_of_slot (warps that reach the grid edge in CTAs of their
//    own); the fused build+backup keeps 32 consecutive cells;
//  * the velocity of every (cell, realisation) is computed once per chunk of
//    realisations (u + sum_k ui_k*Y_k, reference order) into warp-private
//    shared memory and reused by all actions (the reference recomputes it per
//    action); the chunk's mode coefficients are staged once per CTA with
//    asynchronous copies, double-buffered when shared memory allows;
//  * each (cell, action) row histogram lives in a thread-private 8x8 window of
//    16-bit counters in shared memory, placed around the landing cell of the
//    mean flow - no atomics, no sort, exact integer counts.  Samples outside
//    the window are re-run through the full expression; a sample inside the
//    reference's m x m neighbourhood but outside the window switches that row
//    to a dense m*m histogram taken from a global pool (rare);
//  * per-row nonzero bins are emitted in bin order (ascending next state, the
//    order of reduce_kernel) into a staging area at an offset obtained with
//    one atomicAdd per warp (the warp's emission tile = its cell group), with
//    the row's tile-relative offset and R = sumR/nrzns;
//  * K2 scans the tile lengths, K3 moves every tile into canonical CSR order and
//    writes row_ptr.
#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "tile_order.h"

#include "kernels.h"

namespace e2e {

static constexpr int kWin = 8;        // fast window side: bin = li * 8 + lj
static constexpr int kWinBins = kWin * kWin;
static constexpr int kMissBin = kWinBins;  // extra counter row: plain-loop samples that left the window
static constexpr int kNb = 6;         // per-cell obstacle bitmap radius (13 x 13 around S1)
static constexpr int kNbSide = 2 * kNb + 1;
static constexpr int kNbBits = kNbSide * kNbSide;
static constexpr int kNbWords = (kNbBits + 31) / 32;

enum : int { MODE_WINDOW = 0, MODE_FIXED = 1, MODE_DENSE = 2, MODE_LOST = 3 };
enum : int { MASK_OVR = 0, MASK_INWIN = 1, MASK_EDGE = 2, MASK_TERM = 3, MASK_SLOW = 4, MASK_COUNT = 5 };

__device__ __forceinline__ bool bit64(uint64_t m, int b) { return (m >> b) & 1ull; }

// bits lo..hi of a w-bit row (w <= 8), clipped to 0..w-1
__device__ __forceinline__ uint32_t bit_range(int lo, int hi, int w) {
  lo = max(lo, 0);
  hi = min(hi, w - 1);
  return lo > hi ? 0u : (((2u << hi) - 1u) & ~((1u << lo) - 1u));
}

// Realisations per warp-private velocity chunk: BuildArgs::rc (128 for unit
// spacing, whose kernels keep no mask table, 64 otherwise; smaller when shared
// memory is short).  A cell's velocity row has rc + 2 entries: padded so the
// two cells of a warp hit distinct banks, even for 16-byte pair loads.
static constexpr uint32_t kOvrFlag = 0x8000u;   // counter bit 15: bin is obstacle-overridden
static constexpr uint32_t kCountMask = 0x7FFFu;

// Column of a thread in the 16-bit counter rows: lane l of warps 2p and 2p+1
// share the 32-bit word 32p + l, so a warp's 32 lanes hit 32 distinct banks
// whatever bins they update.
__device__ __forceinline__ int counter_col(int warp, int lane) {
  return 64 * (warp >> 1) + 2 * lane + (warp & 1);
}
__host__ __device__ __forceinline__ int counter_log2_stride(int nthr) {
  int l = 6;
  while ((1 << l) < nthr) ++l;
  return l;
}

// Backup of the lane's row (cell, action a) of layer T from its counters:
// Q = R + (sum over entries in column order of fma(count, V[col], acc)) / nrzns
// with R = sumR / nrzns, the arithmetic of the value-iteration sweeps
// (solver_do_backup, src/spvi_2.cu:174-260) on the row the staging path would
// emit; then the first maximum over the cell's action lanes (select_best_action,
// src/spvi_2.cu:93-122: strict '>', NaN never taken, values at or below -1e6
// give -1e6 / -1) and one write of V and the policy per cell.  Entries are
// counted into CTR_STAGE (the model's nnz) per warp.
__device__ __forceinline__ void fused_backup(const BuildArgs& A, int T, int64_t cell, bool valid, bool cvalid,
                                             int a, int lane, int lanes_log2, int mode, float sumR,
                                             const uint16_t* wcol, int log2S, int wi0, int wj0, int i1,
                                             int j1, const uint32_t* dense) {
  const DevProblem& P = A.P;
  const int g = P.g;
  const int64_t nc = (int64_t)g * g;
  // the caller waited for the rows of layer T+1 that it reads (wait_rows)
  const float* Vn = A.V + (int64_t)(T + 1) * nc;
  float acc = 0.f;
  int nnz = 0;
  if (valid) {
    if (mode == MODE_FIXED) {
      acc = fmaf((float)P.nrzns, Vn[cell], acc);
      nnz = 1;
    } else if (mode == MODE_WINDOW) {
      for (int wl = 0; wl < kWinBins; ++wl) {
        const uint32_t c = wcol[wl << log2S] & kCountMask;
        if (c) {
          acc = fmaf((float)c, Vn[(int64_t)(wi0 + wl / kWin) * g + wj0 + wl % kWin], acc);
          ++nnz;
        }
      }
    } else if (mode == MODE_DENSE) {
      for (int b = 0; b < P.m * P.m; ++b) {
        const uint32_t c = dense[b];
        if (c) {
          acc = fmaf((float)c, Vn[(int64_t)(b / P.m + i1 - P.del) * g + b % P.m + j1 - P.del], acc);
          ++nnz;
        }
      }
    }
  }
  const float R = sumR / P.nrzns;  // compute_mean, src/build_model.cu:567
  float q = R + acc / (float)P.nrzns;
  if (!valid || mode == MODE_LOST || isnan(q)) q = -INFINITY;
  int ba = a;
  const int per = 1 << lanes_log2;
  for (int o = per >> 1; o > 0; o >>= 1) {
    const float oq = __shfl_xor_sync(0xffffffffu, q, o);
    const int oa = __shfl_xor_sync(0xffffffffu, ba, o);
    if (oq > q || (oq == q && oa < ba)) {
      q = oq;
      ba = oa;
    }
  }
  for (int o = 16; o > 0; o >>= 1) nnz += __shfl_xor_sync(0xffffffffu, nnz, o);
  if (lane == 0 && nnz) atomicAdd(A.counters + CTR_STAGE, (unsigned long long)nnz);
  if (cvalid && a == 0) {
    const bool ok = q > -1e6f;
    A.V[(int64_t)T * nc + cell] = ok ? q : -1e6f;
    A.pi[(int64_t)T * nc + cell] = ok ? ba : -1;
  }
}

// K1.  Template: CntT = staged count type; UNIT = unit cell spacing.
//
// A CTA owns 32 cells of one layer and all their actions.  Warp w holds
// cells_per_warp = 32/P consecutive cells (P = next power of two >= Na; which
// group, group_of_slot) and lane (c, a) is the row (cell c, action a), so a
// warp computes the velocities of its own cells (u + sum_k ui_k*Y_k, reference
// order) into warp-private shared memory from the chunk's coefficients (staged
// once per CTA; one barrier a chunk with two buffers, two with one), samples
// without further CTA barriers and emits its own rows.
//
// Per row the 8x8 window of the grid around the mean-flow landing cell is
// classified once.  The obstacle override is bit 15 of the bin's 16-bit
// counter; masks kept in shared memory mark `edge` (boundary ring), `term`
// (terminal subgrid) and `slow` bins (outside the m x m neighbourhood, or a
// reward that reads the scalar field).  The reward of a landing is a table
// entry: k = number of r_outbound additions (x clamp, y clamp, edge), terminal
// or not, indexing tab[a] = the reference's float operations evaluated once
// per action (exact for every float input).  Warps without edge/terminal/slow
// bins run a loop that needs none of the masks.  A sample that leaves the
// window (or lands on a slow bin) is only counted; a rescan of the chunk runs
// the full reference expression for it afterwards, so its reward joins the
// row's sum after the chunk's in-window rewards.
//
// FUSED (k_build_fused, one cooperative launch over all layers): instead of
// staging the rows, back them up at once against V of layer t+1 (the rows it
// reads, waited for by wait_rows) and write V, policy of layer t; see
// fused_backup.
// Row stride (floats) of the staged coefficients: a lane reads 8-byte pairs
// of row a + 16r, so an even stride with stride/2 odd (or an odd stride) keeps
// the 16 rows of a warp's loads on distinct banks.
__host__ __device__ __forceinline__ int coeff_stride(int nm) {
  return (nm & 1) ? nm : (((nm >> 1) & 1) ? nm : nm + 2);
}

// min / max that return NaN when either input is NaN (min.NaN / max.NaN):
// a chunk's velocity bounds then become NaN if any velocity is.
__device__ __forceinline__ float fmin_nan(float a, float b) {
  float r;
  asm("min.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ float fmax_nan(float a, float b) {
  float r;
  asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
  return r;
}

// Stages the coefficients of clen realisations (rows of nm floats from src)
// in shared memory, rows ys floats apart: 4-byte asynchronous copies, the
// CTA's threads striding over the elements; one commit group per call.
__device__ __forceinline__ void stage_coeffs(float* ysm, int ys, const float* src, int clen, int nm, int tid,
                                             int nthr) {
  const int n = clen * nm;
  int q = tid / nm, k = tid - q * nm;
  const int dq = nthr / nm, dk = nthr - dq * nm;  // dk < nm
  for (int idx = tid; idx < n; idx += nthr) {
    const uint32_t dst = (uint32_t)__cvta_generic_to_shared(ysm + q * ys + k);
    asm volatile(
        "{\n\t.reg .u64 g;\n\tcvta.to.global.u64 g, %1;\n\tcp.async.ca.shared.global [%0], [g], 4;\n\t}" ::"r"(dst),
        "l"(src + idx)
        : "memory");
    q += dq;
    k += dk;
    if (k >= nm) {
      k -= nm;
      ++q;
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

// Velocity sums of four realisations (staged rows y0 + r * ystep, r = 0..3)
// over NP coefficient pairs: the 4 * NP shared-memory loads are issued before
// the multiply-adds, and each sum is one chain of packed fused multiply-adds in
// mode order.
template <int NP>
__device__ __forceinline__ void vel_pairs4(const float2* md, const float* y0, int ystep, float2& s0,
                                           float2& s1, float2& s2, float2& s3) {
  float2 c[4][NP];
#pragma unroll
  for (int h = 0; h < NP; ++h) {
#pragma unroll
    for (int r = 0; r < 4; ++r) c[r][h] = *reinterpret_cast<const float2*>(y0 + r * ystep + 2 * h);
  }
#pragma unroll
  for (int h = 0; h < NP; ++h) {
    const float2 m0 = md[(2 * h) * 32], m1 = md[(2 * h + 1) * 32];
    s0 = __ffma2_rn(m0, make_float2(c[0][h].x, c[0][h].x), s0);
    s1 = __ffma2_rn(m0, make_float2(c[1][h].x, c[1][h].x), s1);
    s2 = __ffma2_rn(m0, make_float2(c[2][h].x, c[2][h].x), s2);
    s3 = __ffma2_rn(m0, make_float2(c[3][h].x, c[3][h].x), s3);
    s0 = __ffma2_rn(m1, make_float2(c[0][h].y, c[0][h].y), s0);
    s1 = __ffma2_rn(m1, make_float2(c[1][h].y, c[1][h].y), s1);
    s2 = __ffma2_rn(m1, make_float2(c[2][h].y, c[2][h].y), s2);
    s3 = __ffma2_rn(m1, make_float2(c[3][h].y, c[3][h].y), s3);
  }
}

// Fused build+backup: warp 0 waits until every cell of rows lo..hi of layer
// `layer` is backed up (per (layer, grid row) completion counters, released
// by the CTAs of those cells), then the CTA passes a barrier, so every
// thread's later loads of those values are ordered after the writes.  The
// wait is bounded: past A.wait_ns (or a poll limit) it sets FLAG_WAIT_TIMEOUT
// and returns, and once the flag is set every later wait returns at once, so
// the launch drains.  The last layer has no rows: its values are written
// before the launch.
__device__ __forceinline__ void wait_rows(const BuildArgs& A, int layer, int lo, int hi) {
  if (threadIdx.x < 32 && layer <= A.P.nt - 2) {
    const int lane = threadIdx.x;
    const unsigned int target = (unsigned int)A.P.g + A.wait_extra;
    const unsigned int* done = A.layer_done + (int64_t)layer * A.P.g;
    unsigned int* flags = reinterpret_cast<unsigned int*>(A.counters + CTR_FLAGS);
    unsigned long long t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    long long it = 0;
    for (;;) {
      bool ok = true;
      for (int r = lo + lane; r <= hi; r += 32) {
        unsigned int v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(done + r) : "memory");
        ok = ok && v >= target;
      }
      if (__all_sync(0xffffffffu, ok)) break;
      unsigned int f;
      asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(f) : "l"(flags) : "memory");
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      const bool give_up = (f & FLAG_WAIT_TIMEOUT) || ++it > (1ll << 26) || t - t0 > A.wait_ns;
      if (__any_sync(0xffffffffu, give_up)) {
        if (lane == 0) atomicOr(flags, FLAG_WAIT_TIMEOUT);
        break;
      }
      __nanosleep(64);
    }
  }
  __syncthreads();
}

// K1 on one tile (32 cells of layer T and all their actions) by one CTA.
template <typename CntT, bool UNIT, bool FUSED>
__device__ __forceinline__ void build_tile(const BuildArgs& A, unsigned char* smem, const int T, const int tile) {
  const DevProblem& P = A.P;
  const int nthr = blockDim.x;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int nwarps = nthr >> 5;
  const int lanes_log2 = A.lanes_log2;           // P = 1 << lanes_log2 >= na
  const int a = lane & ((1 << lanes_log2) - 1);  // action of this lane
  const int cw = lane >> lanes_log2;             // cell within warp
  const int cl = warp * (32 >> lanes_log2) + cw; // cell within tile (0..31)
  const int g = P.g;
  const int64_t nc = (int64_t)g * g;
  const int64_t c0 = (int64_t)tile * 32;
  // the cells of the tile's warps' groups (group_of_slot), local cell l at
  // cell_tab[l]; the fused pass keeps the identity (its completion counts are
  // per grid row of consecutive cells)
  __shared__ int cell_tab[32];
  if (!FUSED) {
    if (tid < 32) {
      const int cpw_log2 = 5 - lanes_log2;
      const int64_t grp = group_of_slot((int64_t)tile * nwarps + (tid >> cpw_log2), g, 1 << cpw_log2);
      cell_tab[tid] = (int)((grp << cpw_log2) + (tid & ((1 << cpw_log2) - 1)));
    }
    __syncthreads();
  }
  auto cell_of = [&](int l) -> int64_t { return FUSED ? c0 + l : (int64_t)cell_tab[l]; };
  const int64_t cell = cell_of(cl);
  const bool valid = (cell < nc) && (a < P.na);
  const int nm = P.nm;
  const int log2S = counter_log2_stride(nthr);

  const int rc = A.rc, vstride = rc + 2;
  float2* modes = reinterpret_cast<float2*>(smem);                         // nm x 32: (ui, vi)
  float2* velw = modes + nm * 32;                                          // 32 x vstride
  // per-thread bin classes of the general loop (other spacings only): unit
  // spacing derives them from the bin's position where needed
  uint64_t* masks = UNIT ? nullptr : reinterpret_cast<uint64_t*>(velw + 32 * vstride);  // MASK_COUNT x nthr
  uint16_t* win = UNIT ? reinterpret_cast<uint16_t*>(velw + 32 * vstride)
                       : reinterpret_cast<uint16_t*>(masks + MASK_COUNT * nthr);        // 65 x S: bins, miss bin
  __shared__ uint32_t obsmap[32][kNbWords];
  __shared__ float tab[32][8];
  uint16_t* const wcol = win + counter_col(warp, lane);
  float* const ysm = reinterpret_cast<float*>(win + ((size_t)(kWinBins + 1) << log2S));  // rc x coeff_stride(nm)


  // ---- stage the modes of the tile's cells as (ui_k, vi_k) pairs ---------
  for (int idx = tid; idx < 2 * nm * 32; idx += nthr) {
    int k2 = idx >> 5, l = idx & 31;
    int64_t c = cell_of(l);
    float val = 0.f;
    if (c < nc) {
      val = (k2 < nm) ? __ldg(A.F.ui + ((int64_t)T * nm + k2) * nc + c)
                      : __ldg(A.F.vi + ((int64_t)T * nm + (k2 - nm)) * nc + c);
    }
    const int k = k2 < nm ? k2 : k2 - nm;
    reinterpret_cast<float*>(modes)[2 * (k * 32 + l) + (k2 < nm ? 0 : 1)] = val;
  }
  for (int idx = tid; idx < 32 * kNbWords; idx += nthr) obsmap[idx / kNbWords][idx % kNbWords] = 0u;
  const bool late = T > P.nt - 20;
  const bool rad = (P.reward_type == 2 || P.reward_type == 3);
  if (tid < P.na) {
    // landing rewards after k r_outbound additions, then terminal or late, then
    // the step reward: move() + transition_calc's `r += r_step` (:343-354, :533)
    const float Fa = P.ac_speed[tid];
    const float r_step = step_reward(P, Fa, 0.f, 0.f);
    float tk = 0;
    for (int k = 0; k < 4; ++k) {
      float r = tk;
      if (late) r += 0.05 * P.r_out;
      r += r_step;
      tab[tid][k] = r;
      float rt = tk;
      rt += P.r_term;
      rt += r_step;
      tab[tid][4 + k] = rt;
      tk += P.r_out;
    }
  }
  __syncthreads();
  // ---- obstacle override of S1 -> S2 for S2 within 6 cells of S1, per cell
  // (goes_through_obstacle, src/build_model.cu:444-477), shared by the actions.
  // goes_through_obstacle(S1, S2) is the OR, over the obstacle cells o != S1
  // (mask 1 at T or T+1) of the bounding box of S1 and S2, of within_band(o,
  // S1, S2).  The loop runs the other way round: each obstacle cell o within 6
  // cells of S1 tests every S2 whose box with S1 contains it (rows beyond o
  // from S1, or all rows when o is on S1's row; the same for columns), so no
  // box is scanned once per S2; the tests and the bits are the same.
  // The (cell, obstacle) pairs are first collected into a list (in the
  // velocity buffer, unused until the realisation loop), then a warp takes a
  // pair and spreads its tests over the lanes: a thread per pair left every
  // warp waiting on its slowest lane (200x200x120 builder 361 -> 343 ms).
  {
    const int32_t* mT = A.F.mask + (int64_t)T * nc;
    uint16_t* const pairs = reinterpret_cast<uint16_t*>(velw);  // entries c * kNbBits + ob
    const int cap = min(32 * kNbBits, (int)((size_t)32 * vstride * sizeof(float2) / sizeof(uint16_t)));
    __shared__ int npairs;
    for (int s0 = 0; s0 < 32 * kNbBits; s0 += cap) {
      const int s1 = min(s0 + cap, 32 * kNbBits);
      if (tid == 0) npairs = 0;
      __syncthreads();
      for (int i0 = s0; i0 < s1; i0 += nthr) {  // the same trip count in every thread
        const int idx = i0 + tid;
        bool hit = false;
        if (idx < s1) {
          const int c = idx / kNbBits, ob = idx - c * kNbBits;
          const int64_t cc = cell_of(c);
          const int da = ob / kNbSide - kNb, db = ob % kNbSide - kNb;
          if (cc < nc && !(da == 0 && db == 0)) {
            const int ci1 = (int)(cc / g), cj1 = (int)(cc - (int64_t)ci1 * g);
            const int oi = ci1 + da, oj = cj1 + db;
            if (oi >= 0 && oi < g && oj >= 0 && oj < g) {
              const int64_t sp = (int64_t)oj + (int64_t)g * oi;
              hit = __ldg(mT + sp) == 1 || __ldg(mT + nc + sp) == 1;
            }
          }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, hit);
        int at = 0;
        if (lane == 0 && bal) at = atomicAdd(&npairs, __popc(bal));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (hit) pairs[at + __popc(bal & ((1u << lane) - 1u))] = (uint16_t)idx;
      }
      __syncthreads();
      const int n = npairs;
      for (int pi = warp; pi < n; pi += nwarps) {
        const int idx = pairs[pi];
        const int c = idx / kNbBits, ob = idx - c * kNbBits;
        const int64_t cc = cell_of(c);
        const int da = ob / kNbSide - kNb, db = ob % kNbSide - kNb;
        const int ci1 = (int)(cc / g), cj1 = (int)(cc - (int64_t)ci1 * g);
        const int oi = ci1 + da, oj = cj1 + db;
        const int dilo = da > 0 ? da : -kNb, dihi = da < 0 ? da : kNb;
        const int djlo = db > 0 ? db : -kNb, djhi = db < 0 ? db : kNb;
        const int nj = djhi - djlo + 1, ntest = (dihi - dilo + 1) * nj;
        for (int t = lane; t < ntest; t += 32) {
          const int ti = t / nj;
          const int di = dilo + ti, dj = djlo + (t - ti * nj);
          const int i2 = ci1 + di, j2 = cj1 + dj;
          if (i2 < 0 || i2 >= g || j2 < 0 || j2 >= g) continue;
          const int tb = (di + kNb) * kNbSide + (dj + kNb);
          if (within_band(P, oi, oj, ci1, cj1, i2, j2)) atomicOr(&obsmap[c][tb >> 5], 1u << (tb & 31));
        }
      }
      __syncthreads();  // the list is consumed
    }
  }

  // ---- per-row set-up -------------------------------------------------------
  const int i1 = valid ? (int)(cell / g) : 0;
  const int j1 = valid ? (int)(cell - (int64_t)i1 * g) : 0;
  const float x1 = P.xs[j1];
  const float y1 = P.ys[g - 1 - i1];
  const int aa = a < P.na ? a : 0;
  const float F = P.ac_speed[aa];
  const float cs = P.ac_cos[aa];
  const float sn = P.ac_sin[aa];
  const bool cvalid = cell < nc;
  const float u1 = cvalid ? __ldg(A.F.u + (int64_t)T * nc + cell) : 0.f;
  const float v1 = cvalid ? __ldg(A.F.v + (int64_t)T * nc + cell) : 0.f;
  const float rad1 = (cvalid && rad) ? __ldg(A.F.s + (int64_t)T * nc + cell) : 0.f;
  const int W = g < kWin ? g : kWin;

  int mode = MODE_WINDOW;
  float r_fixed = 0.f;
  if (!valid) {
    mode = MODE_FIXED;
  } else if (is_terminal(P, i1, j1)) {
    mode = MODE_FIXED;  // terminal S1: no move, r = 0 (src/build_model.cu:523)
  } else if (__ldg(A.F.mask + (int64_t)T * nc + cell) == 1) {
    mode = MODE_FIXED;  // obstacle S1: no move, r = r_outbound (:542-544)
    r_fixed = P.r_out;
  }
  // obsmap is complete: the pair loop above ends with a barrier
  for (int b = 0; b <= kMissBin; ++b) wcol[b << log2S] = 0;
  int wi0 = 0, wj0 = 0;
  uint64_t ovr = 0, inwin = 0, edge = 0, term = 0, slow = 0;
  if (mode == MODE_WINDOW) {
    int ci, cj;
    land<UNIT>(P, F, cs, sn, u1, v1, x1, y1, ci, cj);
    // window around the mean landing, inside the m x m neighbourhood when the
    // grid allows it, always inside the grid
    wi0 = min(max(ci - (kWin / 2 - 1), i1 - P.del), i1 + P.del - W + 1);
    wj0 = min(max(cj - (kWin / 2 - 1), j1 - P.del), j1 + P.del - W + 1);
    wi0 = min(max(wi0, 0), g - W);
    wj0 = min(max(wj0, 0), g - W);
    // Per window row, the bins (bit lj) in the m x m neighbourhood, on the grid
    // edge, in the terminal subgrid, and obstacle-overridden; the columns of a
    // row are contiguous bits of the obstacle bitmap when the row lies within 6
    // cells of S1, otherwise each bin is tested as before.
    const uint32_t colmask = (1u << W) - 1u;
    const int dj0 = wj0 - j1;
    const uint32_t cols_inw = bit_range(j1 - P.del - wj0, j1 + P.del - wj0, W);
    const uint32_t cols_term = bit_range(P.jt - wj0, P.jt + P.tsg - 1 - wj0, W);
    const uint32_t cols_edge = bit_range(-wj0, -wj0, W) | bit_range(g - 1 - wj0, g - 1 - wj0, W);
    const bool bitmap_cols = dj0 >= -kNb && dj0 + W - 1 <= kNb;
    uint64_t bins = 0;
    for (int li = 0; li < W; ++li) {
      const int i2 = wi0 + li, di = i2 - i1;
      const uint32_t r_inw = (di >= -P.del && di <= P.del) ? cols_inw : 0u;
      const uint32_t r_edge = (i2 == 0 || i2 == g - 1) ? colmask : cols_edge;
      const uint32_t r_term = (i2 >= P.it && i2 < P.it + P.tsg) ? cols_term : 0u;
      uint32_t r_ovr = 0;
      if (di >= -kNb && di <= kNb && bitmap_cols) {
        const int q0 = (di + kNb) * kNbSide + (dj0 + kNb);
        const int w0 = q0 >> 5;
        const uint32_t lo = obsmap[cl][w0], hi = w0 + 1 < kNbWords ? obsmap[cl][w0 + 1] : 0u;
        r_ovr = __funnelshift_r(lo, hi, q0 & 31) & colmask;
      } else {
        for (int lj = 0; lj < W; ++lj) {
          const int j2 = wj0 + lj, dj = j2 - j1;
          bool o;
          if (di >= -kNb && di <= kNb && dj >= -kNb && dj <= kNb) {
            const int nb = (di + kNb) * kNbSide + (dj + kNb);
            o = (obsmap[cl][nb >> 5] >> (nb & 31)) & 1u;
          } else {
            o = through_obstacle(P, A.F.mask, T, i1, j1, i2, j2);
          }
          r_ovr |= (uint32_t)o << lj;
        }
      }
      const int sh = li * kWin;
      bins |= (uint64_t)colmask << sh;
      inwin |= (uint64_t)r_inw << sh;
      edge |= (uint64_t)r_edge << sh;
      term |= (uint64_t)r_term << sh;
      ovr |= (uint64_t)r_ovr << sh;
    }
    slow = rad ? bins : (bins & ~inwin);
    for (uint64_t mo = ovr; mo; mo &= mo - 1) wcol[(__ffsll((long long)mo) - 1) << log2S] = (uint16_t)kOvrFlag;
  }
  if (!UNIT) {
    masks[MASK_OVR * nthr + tid] = ovr;
    masks[MASK_INWIN * nthr + tid] = inwin;
    masks[MASK_EDGE * nthr + tid] = edge;
    masks[MASK_TERM * nthr + tid] = term;
    masks[MASK_SLOW * nthr + tid] = slow;
  }
  // Unit cell spacing: every window row is counted (rewards folded from the
  // counters per bin); a warp whose windows reach the grid's edge ring also
  // counts the clamps of move(), which only samples landing in edge bins can
  // have.  Other spacings take the general loop (per-sample rewards).
  const bool clamp_warp = __any_sync(0xffffffffu, mode == MODE_WINDOW && edge != 0);

  float sumR = 0.f;
  uint32_t n_drop = 0, n_misbin = 0;
  uint32_t* dense = nullptr;
  const int mm = P.m * P.m;
  float2* myvel = velw + cl * vstride;     // this lane's cell
  const int per = 1 << lanes_log2;         // lanes sharing a cell
  // constants of the sample loops, held in registers
  const float xs0 = P.xs0, ysn = P.ysn, axmax = P.axmax, aymax = P.aymax;
  const float xsn = P.xsn, ys0 = P.ys0, dt = P.dt, r_out = P.r_out;
  // the same constants as (x, y) pairs for the packed float2 instructions
  const float2 FF = make_float2(F, F), csn = make_float2(cs, sn), dt2 = make_float2(dt, dt);
  const float2 xy1 = make_float2(x1, y1);
  const float2 sgn = make_float2(1.0f, -1.0f), org = make_float2(-xs0, ysn);
  const bool y_pairs = (nm % 2 == 0);  // staged rows are 8-byte aligned

  // Rewards of the counted (in-window) samples of a row, from its counters.
  // Without a clamp a sample's reward depends only on its bin: r_outbound in an
  // obstacle-overridden bin (src/build_model.cu:538-540), else move()'s edge,
  // terminal and late-time terms plus the step reward (:312-354, :533; the
  // scalar field at the bin for the radiation rewards), evaluated with the
  // reference's float operations; each clamp adds one r_outbound more
  // (:291-310), counted per sample in n_cl.  The row's sum gains count x
  // reward per bin instead of one addition per sample (the reference adds its
  // rewards with float atomics in no fixed order; for integer rewards every
  // partial sum is exact).  Samples in bins outside the m x m neighbourhood
  // are not counted by the reference (their rewards are): they are dropped here.
  int n_cl = 0;
  auto fold_window = [&]() {
    for (int wl = 0; wl < kWinBins; ++wl) {
      uint16_t* p = wcol + (wl << log2S);
      const uint32_t w = *p;
      const uint32_t c = w & kCountMask;
      if (!c) continue;
      // the bin's classes (the masks of the set-up, from its position)
      const int i2 = wi0 + (wl >> 3), j2 = wj0 + (wl & 7);
      const bool in_nb = abs(i2 - i1) <= P.del && abs(j2 - j1) <= P.del;
      float r;
      if (w & kOvrFlag) {
        r = r_out;
      } else {
        const int k = (i2 == 0 || i2 == g - 1 || j2 == 0 || j2 == g - 1) ? 1 : 0;
        const bool tm = is_terminal(P, i2, j2);
        if (!rad) {
          r = tab[aa][(tm ? 4 : 0) + k];
        } else {
          const float rad2 = __ldg(A.F.s + (int64_t)(T + 1) * nc + (int64_t)i2 * g + j2);
          r = k ? r_out : 0.f;
          if (tm) r += P.r_term;
          else if (late) r += 0.05 * P.r_out;
          r += step_reward(P, F, rad1, rad2);
        }
      }
      sumR += (float)c * r;
      if (!in_nb) {
        n_drop += c;
        if (i2 - i1 + P.del < P.m && j2 - j1 + P.del < P.m) n_misbin += c;
        *p = (uint16_t)(w & kOvrFlag);
      }
    }
    sumR += (float)n_cl * r_out;
    n_cl = 0;
  };

  // Full reference expression for one sample (rare): reward, counts, dense
  // switch and drop accounting.
  auto full_sample = [&](float vx, float vy, int i2, int j2) -> float {
    int k2, l2;
    float r;
    move_sample<UNIT>(P, F, cs, sn, vx, vy, x1, y1, late, k2, l2, r);
    float rad2 = 0.f;
    if (rad) rad2 = __ldg(A.F.s + (int64_t)(T + 1) * nc + (int64_t)i2 * g + j2);
    float r_step = step_reward(P, F, rad1, rad2);
    r += r_step;
    const unsigned li = (unsigned)(i2 - wi0), lj = (unsigned)(j2 - wj0);
    if (mode == MODE_WINDOW && li < (unsigned)W && lj < (unsigned)W) {
      const int b = (int)li * kWin + (int)lj;
      // the counter's flag is the bin's obstacle override; in-neighbourhood
      // is the bin's distance from S1
      if (wcol[b << log2S] & kOvrFlag) r = r_out;
      if (abs(i2 - i1) <= P.del && abs(j2 - j1) <= P.del) {
        wcol[b << log2S] += 1;
      } else {
        n_drop++;
        if (i2 - i1 + P.del < P.m && j2 - j1 + P.del < P.m) n_misbin++;
      }
      return r;
    }
    if (through_obstacle(P, A.F.mask, T, i1, j1, i2, j2)) r = r_out;
    const int di = i2 - i1 + P.del, dj = j2 - j1 + P.del;
    if (di >= 0 && di < P.m && dj >= 0 && dj < P.m) {
      if (mode == MODE_WINDOW) {
        // switch this row to a dense m*m histogram from the pool
        if (UNIT) fold_window();  // the window's samples are final
        unsigned long long slot = atomicAdd(A.counters + CTR_POOL, 1ull);
        atomicAdd(A.counters + CTR_OVERFLOW_ROWS, 1ull);
        if (slot < (unsigned long long)A.pool_units) {
          dense = A.pool + slot * (unsigned long long)mm;
          for (int b = 0; b < mm; ++b) dense[b] = 0u;
          for (int wl = 0; wl < kWinBins; ++wl) {
            const uint32_t c = wcol[wl << log2S] & kCountMask;
            if (c) {
              const int ii = wi0 + wl / kWin - i1 + P.del, jj = wj0 + wl % kWin - j1 + P.del;
              dense[ii * P.m + jj] += c;
            }
          }
          mode = MODE_DENSE;
        } else {
          mode = MODE_LOST;
        }
      }
      if (mode == MODE_DENSE) dense[di * P.m + dj] += 1u;
    } else {
      n_drop++;
      if (di < P.m && dj < P.m) n_misbin++;
    }
    return r;
  };

  // ---- realisations in warp-private chunks ----------------------------------
  // The chunk's coefficients (shared by all cells of the layer) are staged
  // once per CTA: the next chunk's copies run while the warps count the
  // current one (each warp loading them from L2: 200x200x120 builder 365 ms,
  // staged: 361 ms).
  // With two buffers (A.ybufs == 2) chunk c+1 is staged into the other buffer
  // as soon as every warp is past chunk c-1, which the barrier opening chunk c
  // shows, so the loop needs that one barrier a chunk; with one buffer a second
  // barrier after the velocity step frees it for the next chunk.
  const int ys = coeff_stride(nm);
  const float* ylayer = A.F.Y + (int64_t)T * P.nrzns * nm;
  const bool two_bufs = A.ybufs == 2;
  const int yalt = two_bufs ? rc * ys : 0;  // offset of the other buffer, toggled by xor
  // velocity bounds of the chunk (plain warps of the unit-spacing staging kernel)
  const bool track = UNIT && !FUSED && !clamp_warp && P.dt > 0.f;
  int yoff = 0;
  stage_coeffs(ysm, ys, ylayer, min(rc, P.nrzns), nm, tid, nthr);
  for (int base = 0; base < P.nrzns; base += rc, yoff ^= yalt) {
    const int clen = min(rc, P.nrzns - base);
    float* const ycur = ysm + yoff;
    asm volatile("cp.async.wait_all;" ::: "memory");
    __syncthreads();  // the chunk's coefficients are staged; the previous chunk is consumed
    if (two_bufs && base + rc < P.nrzns)
      stage_coeffs(ysm + (yoff ^ yalt), ys, ylayer + (int64_t)(base + rc) * nm, min(rc, P.nrzns - base - rc), nm,
                   tid, nthr);
    float2 vlo = make_float2(__int_as_float(0x7f800000), __int_as_float(0x7f800000));  // +inf
    float2 vhi = make_float2(__int_as_float(0xff800000), __int_as_float(0xff800000));  // -inf
    // extract_velocity, src/build_model.cu:389-401: mean + sum over modes, both
    // sums as one chain of packed fused multiply-adds in the reference's order
    if (cvalid) {
      const float2* md = modes + cl;
      const float* yb = ycur;
      const int ystep = per * ys;
      int q = a;
      // four of the lane's realisations at a time: each mode pair read from
      // shared memory feeds four independent chains.  For an even mode count
      // up to ten, vel_pairs4 issues every coefficient load of the four rows
      // before the multiply-adds; the sums keep their order
      for (; q + 3 * per < clen; q += 4 * per) {
        const float* y0 = yb + q * ys;
        float2 s0 = make_float2(0.f, 0.f), s1 = s0, s2 = s0, s3 = s0;
        if (y_pairs && nm <= 10) {  // nm even, rows 8-byte aligned: coefficients two at a time
          switch (nm >> 1) {
            case 5: vel_pairs4<5>(md, y0, ystep, s0, s1, s2, s3); break;
            case 4: vel_pairs4<4>(md, y0, ystep, s0, s1, s2, s3); break;
            case 3: vel_pairs4<3>(md, y0, ystep, s0, s1, s2, s3); break;
            case 2: vel_pairs4<2>(md, y0, ystep, s0, s1, s2, s3); break;
            default: vel_pairs4<1>(md, y0, ystep, s0, s1, s2, s3); break;
          }
        } else if (y_pairs) {
          for (int k = 0; k < nm; k += 2) {
            const float2 m0 = md[k * 32], m1 = md[(k + 1) * 32];
            const float2 c0 = *reinterpret_cast<const float2*>(y0 + k);
            const float2 c1 = *reinterpret_cast<const float2*>(y0 + ystep + k);
            const float2 c2 = *reinterpret_cast<const float2*>(y0 + 2 * ystep + k);
            const float2 c3 = *reinterpret_cast<const float2*>(y0 + 3 * ystep + k);
            s0 = __ffma2_rn(m0, make_float2(c0.x, c0.x), s0);
            s1 = __ffma2_rn(m0, make_float2(c1.x, c1.x), s1);
            s2 = __ffma2_rn(m0, make_float2(c2.x, c2.x), s2);
            s3 = __ffma2_rn(m0, make_float2(c3.x, c3.x), s3);
            s0 = __ffma2_rn(m1, make_float2(c0.y, c0.y), s0);
            s1 = __ffma2_rn(m1, make_float2(c1.y, c1.y), s1);
            s2 = __ffma2_rn(m1, make_float2(c2.y, c2.y), s2);
            s3 = __ffma2_rn(m1, make_float2(c3.y, c3.y), s3);
          }
        } else {
          for (int k = 0; k < nm; k++) {
            const float2 m0 = md[k * 32];
            const float c0 = y0[k], c1 = y0[ystep + k];
            const float c2 = y0[2 * ystep + k], c3 = y0[3 * ystep + k];
            s0 = __ffma2_rn(m0, make_float2(c0, c0), s0);
            s1 = __ffma2_rn(m0, make_float2(c1, c1), s1);
            s2 = __ffma2_rn(m0, make_float2(c2, c2), s2);
            s3 = __ffma2_rn(m0, make_float2(c3, c3), s3);
          }
        }
        const float2 w0 = make_float2(u1 + s0.x, v1 + s0.y), w1 = make_float2(u1 + s1.x, v1 + s1.y);
        const float2 w2 = make_float2(u1 + s2.x, v1 + s2.y), w3 = make_float2(u1 + s3.x, v1 + s3.y);
        myvel[q] = w0;
        myvel[q + per] = w1;
        myvel[q + 2 * per] = w2;
        myvel[q + 3 * per] = w3;
        if (track) {
          vlo.x = fmin_nan(vlo.x, fmin_nan(fmin_nan(w0.x, w1.x), fmin_nan(w2.x, w3.x)));
          vlo.y = fmin_nan(vlo.y, fmin_nan(fmin_nan(w0.y, w1.y), fmin_nan(w2.y, w3.y)));
          vhi.x = fmax_nan(vhi.x, fmax_nan(fmax_nan(w0.x, w1.x), fmax_nan(w2.x, w3.x)));
          vhi.y = fmax_nan(vhi.y, fmax_nan(fmax_nan(w0.y, w1.y), fmax_nan(w2.y, w3.y)));
        }
      }
      for (; q < clen; q += per) {
        const float* y = yb + q * ys;
        float2 sum = make_float2(0.f, 0.f);
        if (y_pairs) {
          for (int k = 0; k < nm; k += 2) {
            const float2 yy = *reinterpret_cast<const float2*>(y + k);
            sum = __ffma2_rn(md[k * 32], make_float2(yy.x, yy.x), sum);
            sum = __ffma2_rn(md[(k + 1) * 32], make_float2(yy.y, yy.y), sum);
          }
        } else {
          for (int k = 0; k < nm; k++) {
            const float yk = y[k];
            sum = __ffma2_rn(md[k * 32], make_float2(yk, yk), sum);
          }
        }
        const float2 w0 = make_float2(u1 + sum.x, v1 + sum.y);
        myvel[q] = w0;
        if (track) {
          vlo = make_float2(fmin_nan(vlo.x, w0.x), fmin_nan(vlo.y, w0.y));
          vhi = make_float2(fmax_nan(vhi.x, w0.x), fmax_nan(vhi.y, w0.y));
        }
      }
    }
    // Plain warps of the staging kernel: does every sample of the chunk land in
    // its row's window?  The snapping chain (advection, offset, two round-down
    // adds) is monotone in each velocity component (every step rounds a
    // function increasing in the component, x increasing and y decreasing, for
    // dt > 0), so the bins of the chunk's samples lie between those of the
    // bounding box's corners (vx min, vy max) and (vx max, vy min) of the cell's
    // velocities (a NaN velocity makes the bounds NaN: never in the window).
    // If the corners are in the window for every counting lane of the warp,
    // the chunk runs the loop without the window test and the miss counter.
    bool in_win = false;
    if (track) {
      for (int o = 1; o < per; o <<= 1) {
        vlo.x = fmin_nan(vlo.x, __shfl_xor_sync(0xffffffffu, vlo.x, o));
        vlo.y = fmin_nan(vlo.y, __shfl_xor_sync(0xffffffffu, vlo.y, o));
        vhi.x = fmax_nan(vhi.x, __shfl_xor_sync(0xffffffffu, vhi.x, o));
        vhi.y = fmax_nan(vhi.y, __shfl_xor_sync(0xffffffffu, vhi.y, o));
      }
      bool ok = true;
      if (mode == MODE_WINDOW) {
        const uint32_t M = 0x4B400000u;
        const float2 magic = make_float2(12582912.0f - (float)wj0, 12582912.0f - (float)wi0);
        const float2 half = make_float2(0.5f, 0.5f);
        const float2 tl = __fadd2_rd(
            __fadd2_rd(__ffma2_rn(advect2(FF, csn, make_float2(vlo.x, vhi.y), dt2, xy1), sgn, org), half), magic);
        const float2 th = __fadd2_rd(
            __fadd2_rd(__ffma2_rn(advect2(FF, csn, make_float2(vhi.x, vlo.y), dt2, xy1), sgn, org), half), magic);
        ok = ((__float_as_uint(tl.x) ^ M) | (__float_as_uint(tl.y) ^ M) | (__float_as_uint(th.x) ^ M) |
              (__float_as_uint(th.y) ^ M)) < (uint32_t)kWin;
      }
      in_win = __all_sync(0xffffffffu, ok);
    }
    if (!two_bufs) {
      __syncthreads();  // every warp has read the chunk's coefficients
      if (base + rc < P.nrzns)
        stage_coeffs(ysm, ys, ylayer + (int64_t)(base + rc) * nm, min(rc, P.nrzns - base - rc), nm, tid, nthr);
    }
    if (mode == MODE_FIXED) {
      for (int q = 0; q < clen; ++q) sumR += r_fixed;
    } else if (mode == MODE_WINDOW) {
      int n_out = 0;
      if (UNIT) {
        // counts only: the rewards are folded from the counters at the end, a
        // sample that leaves the window counts in the miss bin
        // The window origin is folded into the rounding constant: the bits of
        // RD(w + 1.5*2^23 - wj0) are 0x4B400000 + lj (exact while |w - wj0| <
        // 2^22, the floats there being the integers), so one three-input logic
        // op tests both coordinates, and the counter's 32-bit shared address
        // is base + (8*by + bx) << sh with the offset 9*0x4B400000 folded into
        // the base, modulo 2^32 (200x200x120 builder 413 -> 409 ms).
        const uint32_t M = 0x4B400000u;
        const float2 magic = make_float2(12582912.0f - (float)wj0, 12582912.0f - (float)wi0);
        const uint32_t sh = (uint32_t)log2S + 1u;  // bytes per bin row, log2
        const uint32_t base_adj = (uint32_t)__cvta_generic_to_shared(wcol) - ((9u * M) << sh);
        const uint32_t miss_idx = 9u * M + (uint32_t)kMissBin;
        // one sample at window-relative snapping coordinates d: its window bin
        // (or the miss bin) counter incremented; returns the counter's value
        // before
        auto bump = [&](float2 d, bool& inw) -> uint32_t {
          const float2 w = __fadd2_rd(d, make_float2(0.5f, 0.5f));  // round_half_up_index
          const float2 t = __fadd2_rd(w, magic);
          const uint32_t bx = __float_as_uint(t.x), by = __float_as_uint(t.y);
          inw = ((bx ^ M) | (by ^ M)) < (uint32_t)kWin;
          const uint32_t addr = base_adj + ((inw ? (by << 3) + bx : miss_idx) << sh);
          unsigned short v;
          asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(addr));
          const unsigned short v1 = (unsigned short)(v + 1);
          asm volatile("st.shared.u16 [%0], %1;" ::"r"(addr), "h"(v1));
          return v;
        };
        // (xnew - xs0, -(ynew - ysn)) without the domain clamps: in a warp
        // whose windows hold no edge cell a sample the clamps would move lands
        // outside the window either way (unclamped its index is below 0 or
        // above g-1; a NaN or a value beyond 2^22 gives bits far from
        // 0x4B400000) and is taken again by the rescan below
        auto count_sample = [&](float2 vv) {
          const float2 xy = advect2(FF, csn, vv, dt2, xy1);  // move(), src/build_model.cu:284-289
          bool inw;
          bump(__ffma2_rn(xy, sgn, org), inw);
        };
        // a warp whose windows hold edge bins: the domain clamps applied to the
        // snapping coordinates (land_unit), and each clamp of a counted sample
        // outside an obstacle-overridden bin adds one r_outbound
        auto count_sample_clamp = [&](float2 vv) {
          const float2 xy = advect2(FF, csn, vv, dt2, xy1);
          const float2 d = __ffma2_rn(xy, sgn, org);
          bool inw;
          const uint32_t v =
              bump(make_float2(fminf(fmaxf(d.x, 0.0f), axmax), fminf(fmaxf(d.y, 0.0f), aymax)), inw);
          const bool add = inw && !(v & kOvrFlag);
          n_cl += (add && (xy.x > xsn || xy.x < xs0)) ? 1 : 0;
          n_cl += (add && (xy.y > ysn || xy.y < ys0)) ? 1 : 0;
        };
        if (clamp_warp) {
#pragma unroll 8
          for (int q = 0; q < clen; ++q) count_sample_clamp(myvel[q]);
        } else if constexpr (FUSED) {
          // one realisation a load: the fused instance measured 444 ms with
          // the pairs below and 419 ms without them (200x200x120)
#pragma unroll 16
          for (int q = 0; q < clen; ++q) count_sample(myvel[q]);
        } else if (in_win) {
          // every sample of the chunk is in the window (bounding box above): the
          // bin is the low six bits of (by << 3) + bx (the 0x4B400000 offsets
          // have none), masked so that the address stays in the lane's counters
          const uint32_t wsh = (uint32_t)__cvta_generic_to_shared(wcol);
          const uint32_t row_bytes = 1u << sh;
          auto count_in_window = [&](float2 vv) {
            const float2 xy = advect2(FF, csn, vv, dt2, xy1);
            const float2 w = __fadd2_rd(__ffma2_rn(xy, sgn, org), make_float2(0.5f, 0.5f));
            const float2 t = __fadd2_rd(w, magic);
            const uint32_t b = ((__float_as_uint(t.y) << 3) + __float_as_uint(t.x)) & 63u;
            const uint32_t addr = wsh + b * row_bytes;
            unsigned short v;
            asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(addr));
            const unsigned short v1 = (unsigned short)(v + 1);
            asm volatile("st.shared.u16 [%0], %1;" ::"r"(addr), "h"(v1));
          };
          int q = 0;
#pragma unroll 8
          for (; q + 1 < clen; q += 2) {
            const float4 v2 = *reinterpret_cast<const float4*>(myvel + q);
            count_in_window(make_float2(v2.x, v2.y));
            count_in_window(make_float2(v2.z, v2.w));
          }
          if (q < clen) count_in_window(myvel[q]);
        } else {
          // two realisations a 16-byte load (the velocity rows have an even
          // stride): 200x200x120 builder 409 -> 393 ms
          int q = 0;
#pragma unroll 8
          for (; q + 1 < clen; q += 2) {
            const float4 v2 = *reinterpret_cast<const float4*>(myvel + q);
            count_sample(make_float2(v2.x, v2.y));
            count_sample(make_float2(v2.z, v2.w));
          }
          if (q < clen) count_sample(myvel[q]);
        }
        asm volatile("" ::: "memory");  // the counters are read below
        uint16_t* mp = wcol + (kMissBin << log2S);
        n_out = *mp;
        if (n_out) *mp = 0;
      } else {
        // general cell spacing: the reference's remainderf snapping and a
        // reward per sample
        const uint64_t m_edge = masks[MASK_EDGE * nthr + tid];
        const uint64_t m_term = masks[MASK_TERM * nthr + tid];
        const uint64_t m_slow = masks[MASK_SLOW * nthr + tid];
#pragma unroll 8
        for (int q = 0; q < clen; ++q) {
          const float2 vv = myvel[q];
          const float2 xy = advect2(FF, csn, vv, dt2, xy1);
          const float xnew = xy.x, ynew = xy.y;
          const int kcl = ((xnew > xsn) || (xnew < xs0) ? 1 : 0) + ((ynew > ysn) || (ynew < ys0) ? 1 : 0);
          int i2, j2;
          land<UNIT>(P, F, cs, sn, vv.x, vv.y, x1, y1, i2, j2);
          const int li = i2 - wi0, lj = j2 - wj0;
          const bool inw = (unsigned)(li | lj) < (unsigned)kWin;
          const int b = inw ? (li << 3) + lj : 0;
          const bool fast = inw && !bit64(m_slow, b);
          uint16_t* wp = wcol + (b << log2S);
          const uint32_t w = *wp;
          const int k = kcl + (bit64(m_edge, b) ? 1 : 0);
          float r = tab[aa][(bit64(m_term, b) ? 4 : 0) + k];
          if (w & kOvrFlag) r = r_out;
          *wp = (uint16_t)(fast ? w + 1 : w);
          const float s2 = sumR + r;
          sumR = fast ? s2 : sumR;
          n_out += fast ? 0 : 1;
        }
      }
      if (n_out) {
        // rescan: the chunk's samples that left the window or (general loop)
        // hit a slow bin.  With unit spacing the counting loops counted exactly
        // the samples whose clamped landing (land_unit) is in the window: the
        // edge warps clamp, and in the others an in-window sample is never
        // clamped
        const uint64_t m_slow = UNIT ? 0ull : masks[MASK_SLOW * nthr + tid];
        for (int q = 0; q < clen; ++q) {
          const float2 vv = myvel[q];
          int i2, j2;
          land<UNIT>(P, F, cs, sn, vv.x, vv.y, x1, y1, i2, j2);
          const int li = i2 - wi0, lj = j2 - wj0;
          const bool inw = (unsigned)(li | lj) < (unsigned)kWin;
          if (inw && !bit64(m_slow, (li << 3) + lj)) continue;
          const float r = full_sample(vv.x, vv.y, i2, j2);
          sumR += r;
        }
      }
    } else if (mode == MODE_DENSE) {
      for (int q = 0; q < clen; ++q) {
        const float2 vv = myvel[q];
        int i2, j2;
        land<UNIT>(P, F, cs, sn, vv.x, vv.y, x1, y1, i2, j2);
        const float r = full_sample(vv.x, vv.y, i2, j2);
        sumR += r;
      }
    }
  }
  if (UNIT && mode == MODE_WINDOW) fold_window();
  if (n_drop) atomicAdd(A.counters + CTR_DROPPED, (unsigned long long)n_drop);
  if (n_misbin) atomicAdd(A.counters + CTR_MISBIN, (unsigned long long)n_misbin);
  if (mode == MODE_LOST) atomicOr(reinterpret_cast<unsigned int*>(A.counters + CTR_FLAGS), FLAG_POOL_EXHAUSTED);

  if (FUSED) {
    // the backup reads layer T+1 within the rows' m x m neighbourhoods and
    // 8 x 8 windows: rows of the tile's cells +- max(del, 7)
    const int64_t c_last = min(c0 + 31, nc - 1);
    const int r0 = (int)(c0 / g), r1 = (int)(c_last / g), reach = max(P.del, kWin - 1);
    wait_rows(A, T + 1, max(r0 - reach, 0), min(r1 + reach, g - 1));
    fused_backup(A, T, cell, valid, cvalid, a, lane, lanes_log2, mode, sumR, wcol, log2S, wi0, wj0, i1, j1,
                 dense);
    __syncthreads();  // every row of the tile is backed up
    if (tid == 0) {
      __threadfence();
      for (int r = r0; r <= r1; ++r) {  // the tile's cells in each grid row it spans
        const int64_t lo = max(c0, (int64_t)r * g), hi = min(c_last, (int64_t)(r + 1) * g - 1);
        asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(A.layer_done + (int64_t)T * g + r),
                     "r"((unsigned int)(hi - lo + 1))
                     : "memory");
      }
    }
    return;
  }

  // ---- per-warp emission: row lengths, warp scan, one atomicAdd -----------
  int nnz = 0;
  if (valid) {
    if (mode == MODE_FIXED) {
      nnz = 1;
    } else if (mode == MODE_WINDOW) {
      for (int wl = 0; wl < kWinBins; ++wl) nnz += (wcol[wl << log2S] & kCountMask) != 0;
    } else if (mode == MODE_DENSE) {
      for (int b = 0; b < mm; ++b) nnz += dense[b] != 0u;
    }
  }
  // lane order = (cell, action) order of the warp's rows; padding lanes add 0
  int incl = nnz;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t2 = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t2;
  }
  const int total = __shfl_sync(0xffffffffu, incl, 31);
  unsigned long long wbase = 0;
  if (lane == 0) {
    wbase = atomicAdd(A.counters + CTR_STAGE, (unsigned long long)total);
    const int64_t wt = (int64_t)T * A.tiles_per_layer * nwarps + (cell_tab[warp << (5 - A.lanes_log2)] >> (5 - A.lanes_log2));
    A.tile_base[wt] = (int64_t)wbase;
    A.tile_len[wt] = total;
  }
  wbase = __shfl_sync(0xffffffffu, wbase, 0);
  if (!valid) return;
  const int excl = incl - nnz;
  // the lane's cell again from the group table (a shared-memory load, not a
  // register held through the sample loops)
  const int64_t cell_e = cell_of(cl);
  const int64_t grow = ((int64_t)T * nc + cell_e) * P.na + a;
  A.row_off[grow] = (uint32_t)excl;
  A.R[grow] = sumR / P.nrzns;  // compute_mean, src/build_model.cu:567
  if (A.sumR) A.sumR[grow] = sumR;  // kept for re-targeting (served requests)
  if (mode == MODE_LOST) return;
  unsigned long long off = wbase + (unsigned long long)excl;
  if (off + (unsigned long long)nnz > (unsigned long long)A.stage_cap) return;  // host re-runs
  CntT* scnt = reinterpret_cast<CntT*>(A.stage_cnt);
  const int64_t next_layer = (int64_t)(T + 1) * nc;
  if (mode == MODE_FIXED) {
    A.stage_col[off] = (int32_t)(next_layer + cell_e);
    scnt[off] = (CntT)P.nrzns;
  } else if (mode == MODE_WINDOW) {
    for (int wl = 0; wl < kWinBins; ++wl) {
      const uint32_t c = wcol[wl << log2S] & kCountMask;
      if (c) {
        const int i2 = wi0 + wl / kWin, j2 = wj0 + wl % kWin;
        A.stage_col[off] = (int32_t)(next_layer + (int64_t)i2 * g + j2);
        scnt[off] = (CntT)c;
        ++off;
      }
    }
  } else {  // MODE_DENSE: bins in reference order
    for (int b = 0; b < mm; ++b) {
      const uint32_t c = dense[b];
      if (c) {
        const int i2 = b / P.m + i1 - P.del, j2 = b % P.m + j1 - P.del;
        A.stage_col[off] = (int32_t)(next_layer + (int64_t)i2 * g + j2);
        scnt[off] = (CntT)c;
        ++off;
      }
    }
  }
}

// K1 over a grid of (tile, layer - t0) CTAs.
template <typename CntT, bool UNIT>
__global__ void __launch_bounds__(1024) k_build_tiles(BuildArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  build_tile<CntT, UNIT, false>(A, smem, A.t0 + (int)blockIdx.y, (int)blockIdx.x);
}

// Fused build+backup of all layers in one cooperative launch.  Tiles are
// numbered g = 0, 1, ... with layer nt-2-g/tiles_per_layer, and a CTA that is
// ready takes the next number from a counter (CTR_NEXT_TILE); a tile samples,
// waits for the layer after its own (wait_rows), backs its rows up and counts
// itself done.  Every tile of layer t+1 has a smaller number than every tile
// of layer t and numbers are taken in increasing order by resident CTAs (a
// cooperative launch), so by induction over g every awaited tile has been
// taken and finishes: the waits end.  A tile waits only for the rows of layer
// t+1 its backup reads (its cells' rows +- max(del, 7)), which were taken
// about a layer's worth of tiles before it.  Sampling needs no values, so a
// layer's sampling overlaps the completion of the layer after it, with no
// launch boundary between layers.  (Fixed assignment, CTA b taking g = b, b + grid,
// ..., let slow CTAs fall ever further behind and the others wait for them at
// every layer: 400 ms on c2 against 367 ms with one launch per layer.)
template <typename CntT, bool UNIT>
__global__ void __launch_bounds__(1024) k_build_fused(BuildArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long taken;
  const int64_t tpl = A.tiles_per_layer;
  const int64_t total = (int64_t)(A.P.nt - 1) * tpl;
  for (;;) {
    if (threadIdx.x == 0) taken = (long long)atomicAdd(A.counters + CTR_NEXT_TILE, 1ull);
    __syncthreads();
    const int64_t g = taken;
    if (g >= total) break;
    const int L = (int)(g / tpl);
    build_tile<CntT, UNIT, true>(A, smem, A.P.nt - 2 - L, (int)(g - (int64_t)L * tpl));
    __syncthreads();  // the next tile reuses the shared memory (and `taken`)
  }
}

// K2: exclusive scan of the tile lengths (tile order == row order), in three
// steps: per-block sums, one block scanning the block sums, per-block scans.
static constexpr int kScanBlock = 1024;

__global__ void k_scan_sums(const int32_t* __restrict__ len, int64_t n, int64_t* __restrict__ sums) {
  __shared__ int64_t red[32];
  const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
  int64_t v = i < n ? len[i] : 0;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    int64_t w = red[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if (threadIdx.x == 0) sums[blockIdx.x] = w;
  }
}

__global__ void k_scan_block_sums(int64_t* sums, int64_t nb, int64_t* total) {
  __shared__ int64_t part[1024];
  const int tid = threadIdx.x;
  const int64_t per = (nb + 1023) / 1024;
  const int64_t b = min((int64_t)tid * per, nb), e = min(b + per, nb);
  int64_t s = 0;
  for (int64_t i = b; i < e; ++i) s += sums[i];
  part[tid] = s;
  __syncthreads();
  if (tid == 0) {
    int64_t run = 0;
    for (int k = 0; k < 1024; ++k) {
      int64_t x = part[k];
      part[k] = run;
      run += x;
    }
    *total = run;
  }
  __syncthreads();
  int64_t run = part[tid];
  for (int64_t i = b; i < e; ++i) {
    int64_t x = sums[i];
    sums[i] = run;
    run += x;
  }
}

__global__ void k_scan_finish(const int32_t* __restrict__ len, int64_t n,
                              const int64_t* __restrict__ sums, int64_t* __restrict__ out) {
  __shared__ int64_t wsum[32];
  const int64_t i = (int64_t)blockIdx.x * kScanBlock + threadIdx.x;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int64_t v = i < n ? len[i] : 0;
  int64_t incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    int64_t t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    int64_t x = wsum[lane];
    int64_t xi = x;
    for (int o = 1; o < 32; o <<= 1) {
      int64_t t = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += t;
    }
    wsum[lane] = xi - x;
  }
  __syncthreads();
  if (i < n) out[i] = sums[blockIdx.x] + wsum[w] + incl - v;
}

// K3: one warp per tile (the rows of one builder warp): move the tile's
// entries from staging to their canonical position and write row_ptr.
template <typename CntT, typename PtrT>
__global__ void k_assemble(AssembleArgs A) {
  const int lane = threadIdx.x & 31;
  const int64_t tile = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (tile >= A.n_tiles) return;
  const int64_t src = A.tile_base[tile];
  const int64_t dst = A.canon[tile];
  const int len = A.tile_len[tile];
  const int32_t* __restrict__ scol = A.stage_col + src;
  const CntT* __restrict__ scnt = reinterpret_cast<const CntT*>(A.stage_cnt) + src;
  int32_t* __restrict__ dcol = A.col + dst;
  CntT* __restrict__ dcnt = reinterpret_cast<CntT*>(A.cnt) + dst;
  for (int k = lane; k < len; k += 32) {
    dcol[k] = scol[k];
    dcnt[k] = scnt[k];
  }
  const int64_t layer = tile / A.tiles_per_layer;
  const int64_t tl = tile - layer * A.tiles_per_layer;
  const int64_t cb = tl * A.cells_per_tile;
  const int64_t ce = min(cb + A.cells_per_tile, A.ncells);
  PtrT* rp = reinterpret_cast<PtrT*>(A.row_ptr);
  if (cb < ce) {
    const int64_t r0 = (layer * A.ncells + cb) * A.na;
    const int64_t r1 = (layer * A.ncells + ce) * A.na;
    for (int64_t r = r0 + lane; r < r1; r += 32) rp[r] = (PtrT)(dst + A.row_off[r]);
  }
  if (tile == A.n_tiles - 1 && lane == 0) rp[A.n_rows] = (PtrT)A.total_nnz;
}

// Device cosf/sinf of the headings: the values move() multiplies by F
// (src/build_model.cu:284-285 evaluates them per sample with the same functions).
__global__ void k_action_trig(const float* angle, int n, float* cosv, float* sinv) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    cosv[k] = cosf(angle[k]);
    sinv[k] = sinf(angle[k]);
  }
}

// ---- launch wrappers ---------------------------------------------------------

int build_lanes_log2(int na) {
  int l = 0;
  while ((1 << l) < na) ++l;
  return l;
}

size_t build_smem_bytes(int na, int nm, int rc, bool unit, int ybufs) {
  const int nthr = 32 << build_lanes_log2(na);
  return (size_t)2 * nm * 32 * sizeof(float) + (size_t)32 * (rc + 2) * sizeof(float2) +
         (unit ? 0 : (size_t)MASK_COUNT * nthr * sizeof(uint64_t)) +
         (size_t)(kWinBins + 1) * ((size_t)1 << counter_log2_stride(nthr)) * sizeof(uint16_t) +
         (size_t)ybufs * rc * coeff_stride(nm) * sizeof(float);
}

int build_ctas_per_sm(int na, size_t smem, bool unit) {
  int dev = 0, smem_sm = 0, reserved = 0, regs_sm = 0, thr_sm = 0;
  // a failed query answers 0 and leaves no error behind for the next launch check
  auto none = []() {
    cudaGetLastError();
    return 0;
  };
  if (cudaGetDevice(&dev) != cudaSuccess) return none();
  if (cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess)
    return none();
  const int nthr = 32 << build_lanes_log2(na);
  int best = thr_sm / nthr;
  // the staging kernel with 16- and 32-bit counts, and the fused kernel
  cudaFuncAttributes fa[3];
  cudaError_t e = unit ? cudaFuncGetAttributes(&fa[0], k_build_tiles<uint16_t, true>)
                       : cudaFuncGetAttributes(&fa[0], k_build_tiles<uint16_t, false>);
  if (e != cudaSuccess) return none();
  e = unit ? cudaFuncGetAttributes(&fa[1], k_build_tiles<uint32_t, true>)
           : cudaFuncGetAttributes(&fa[1], k_build_tiles<uint32_t, false>);
  if (e != cudaSuccess) return none();
  e = unit ? cudaFuncGetAttributes(&fa[2], k_build_fused<uint32_t, true>)
           : cudaFuncGetAttributes(&fa[2], k_build_fused<uint32_t, false>);
  if (e != cudaSuccess) return none();
  for (const cudaFuncAttributes& f : fa) {
    const size_t per_cta = smem + f.sharedSizeBytes + (size_t)reserved;
    best = std::min(best, (int)((size_t)smem_sm / per_cta));
    if (f.numRegs > 0) best = std::min(best, regs_sm / (f.numRegs * nthr));
  }
  return best;
}

// the dynamic shared-memory cap of a kernel only grows: builds on other host
// threads may be launching it with a larger need at the same time
template <typename K>
static cudaError_t raise_smem_cap(K kern, size_t sm, int* cap_set, std::mutex& mu) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if (dev >= 0 && dev < 64 && (int)sm > cap_set[dev]) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    cap_set[dev] = (int)sm;
  }
  return cudaSuccess;
}

template <typename CntT, bool UNIT>
static cudaError_t launch_one(const BuildArgs& A, int n_layers, cudaStream_t st) {
  dim3 grid((unsigned)A.tiles_per_layer, (unsigned)n_layers);
  dim3 block((unsigned)(32u << A.lanes_log2));
  const size_t sm = build_smem_bytes(A.P.na, A.P.nm, A.rc, UNIT, A.ybufs);
  static std::mutex mu;
  static int cap_set[64] = {};
  cudaError_t e = raise_smem_cap(k_build_tiles<CntT, UNIT>, sm, cap_set, mu);
  if (e != cudaSuccess) return e;
  k_build_tiles<CntT, UNIT><<<grid, block, sm, st>>>(A);
  return cudaGetLastError();
}

template <bool UNIT>
static cudaError_t launch_fused(const BuildArgs& A, cudaStream_t st, int* grid_out) {
  auto kern = k_build_fused<uint32_t, UNIT>;
  const int threads = 32 << A.lanes_log2;
  const size_t sm = build_smem_bytes(A.P.na, A.P.nm, A.rc, UNIT, A.ybufs);
  static std::mutex mu;
  static int cap_set[64] = {};
  cudaError_t e = raise_smem_cap(kern, sm, cap_set, mu);
  if (e != cudaSuccess) return e;
  int dev = 0, per_sm = 0, sms = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, sm)) != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int64_t total = (int64_t)(A.P.nt - 1) * A.tiles_per_layer;
  const unsigned grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(total, (int64_t)per_sm * sms));
  if (grid_out) *grid_out = (int)grid;
  BuildArgs B = A;
  void* args[] = {&B};
  return cudaLaunchCooperativeKernel((const void*)kern, dim3(grid), dim3((unsigned)threads), args, sm, st);
}

cudaError_t launch_build_tiles(const BuildArgs& A, int count_bits, int n_layers,
                               cudaStream_t st) {
  const bool unit = A.P.unit_step != 0;
  if (count_bits == 16) return unit ? launch_one<uint16_t, true>(A, n_layers, st)
                                    : launch_one<uint16_t, false>(A, n_layers, st);
  return unit ? launch_one<uint32_t, true>(A, n_layers, st) : launch_one<uint32_t, false>(A, n_layers, st);
}

cudaError_t launch_build_fused(const BuildArgs& A, cudaStream_t st, int* grid) {
  return A.P.unit_step != 0 ? launch_fused<true>(A, st, grid) : launch_fused<false>(A, st, grid);
}

cudaError_t launch_scan_tiles(const int32_t* tile_len, int64_t n_tiles, int64_t* canon,
                              int64_t* total, int64_t* block_sums, cudaStream_t st) {
  const int64_t nb = (n_tiles + kScanBlock - 1) / kScanBlock;
  if (nb == 0) return cudaSuccess;
  k_scan_sums<<<(unsigned)nb, kScanBlock, 0, st>>>(tile_len, n_tiles, block_sums);
  k_scan_block_sums<<<1, 1024, 0, st>>>(block_sums, nb, total);
  k_scan_finish<<<(unsigned)nb, kScanBlock, 0, st>>>(tile_len, n_tiles, block_sums, canon);
  return cudaGetLastError();
}

cudaError_t launch_assemble(const AssembleArgs& A, int count_bits, int index_bits,
                            cudaStream_t st) {
  dim3 grid((unsigned)((A.n_tiles + 7) / 8)), block(256);
  if (A.n_tiles == 0) return cudaSuccess;
  if (count_bits == 16 && index_bits == 32) k_assemble<uint16_t, int32_t><<<grid, block, 0, st>>>(A);
  else if (count_bits == 16) k_assemble<uint16_t, int64_t><<<grid, block, 0, st>>>(A);
  else if (index_bits == 32) k_assemble<uint32_t, int32_t><<<grid, block, 0, st>>>(A);
  else k_assemble<uint32_t, int64_t><<<grid, block, 0, st>>>(A);
  return cudaGetLastError();
}

cudaError_t launch_action_trig(const float* angle, int n, float* cosv, float* sinv,
                               cudaStream_t st) {
  k_action_trig<<<(n + 127) / 128, 128, 0, st>>>(angle, n, cosv, sinv);
  return cudaGetLastError();
}

}  // namespace e2e
