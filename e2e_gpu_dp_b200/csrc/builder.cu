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
//  * a CTA owns a tile of 32 consecutive cells of one layer and all actions
//    (warp w = action w, lane = cell), i.e. a contiguous range of model rows;
//  * the velocity of every (cell, realisation) is computed once per CTA chunk
//    (u + sum_k ui_k*Y_k, reference order) into shared memory and reused by all
//    actions (the reference recomputes it per action);
//  * each (cell, action) row histogram lives in a thread-private 7x7 window of
//    16-bit counters in shared memory, placed around the landing cell of the
//    mean flow - no atomics, no sort, exact integer counts.  A sample outside
//    the window but inside the reference's m x m neighbourhood switches that
//    row to a dense m*m histogram taken from a global pool (rare);
//  * per-row nonzero bins are emitted in bin order (ascending next state, the
//    order of reduce_kernel) into a staging area at a tile offset obtained with
//    one atomicAdd per CTA, with the row's tile-relative offset and R = sumR/nrzns;
//  * K2 scans the tile lengths, K3 moves every tile into canonical CSR order and
//    writes row_ptr.
#include "common.cuh"
#include "kernels.h"

namespace e2e {

static constexpr int kWin = 7;            // fast window side
static constexpr int kWinWords = 25;      // ceil(49 / 2) packed 16-bit counters

enum : int { MODE_WINDOW = 0, MODE_FIXED = 1, MODE_DENSE = 2, MODE_LOST = 3 };

template <typename CntT>
__global__ void __launch_bounds__(1024) k_build_tiles(BuildArgs A) {
  extern __shared__ __align__(16) unsigned char smem[];
  const DevProblem& P = A.P;
  const int nthr = blockDim.x;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int a = tid >> 5;
  const int nwarps = nthr >> 5;
  const int T = A.t0 + blockIdx.y;
  const int g = P.g;
  const int64_t nc = (int64_t)g * g;
  const int64_t c0 = (int64_t)blockIdx.x * 32;
  const int64_t cell = c0 + lane;
  const bool valid = cell < nc;
  const int nm = P.nm;

  float2* vel = reinterpret_cast<float2*>(smem);                     // rc x 32
  float* modes = reinterpret_cast<float*>(vel + (size_t)A.rc * 32);  // 2*nm x 32
  uint32_t* win = reinterpret_cast<uint32_t*>(modes + 2 * nm * 32);  // kWinWords x nthr
  int* scan = reinterpret_cast<int*>(win + kWinWords * nthr);        // nthr
  __shared__ int warp_tot[32];
  __shared__ unsigned long long tile_base_sh;

  // ---- stage the modes of the tile's cells (ui then vi) -------------------
  for (int idx = tid; idx < 2 * nm * 32; idx += nthr) {
    int k2 = idx >> 5, l = idx & 31;
    int64_t c = c0 + l;
    float val = 0.f;
    if (c < nc) {
      val = (k2 < nm) ? __ldg(A.F.ui + ((int64_t)T * nm + k2) * nc + c)
                      : __ldg(A.F.vi + ((int64_t)T * nm + (k2 - nm)) * nc + c);
    }
    modes[idx] = val;
  }

  // ---- per-row set-up -------------------------------------------------------
  const int i1 = valid ? (int)(cell / g) : 0;
  const int j1 = valid ? (int)(cell - (int64_t)i1 * g) : 0;
  const float x1 = P.xs[j1];
  const float y1 = P.ys[g - 1 - i1];
  const float F = P.ac_speed[a];
  const float cs = P.ac_cos[a];
  const float sn = P.ac_sin[a];
  const bool late = T > P.nt - 20;
  const bool rad = (P.reward_type == 2 || P.reward_type == 3);
  const float u1 = valid ? __ldg(A.F.u + (int64_t)T * nc + cell) : 0.f;
  const float v1 = valid ? __ldg(A.F.v + (int64_t)T * nc + cell) : 0.f;
  const float rad1 = (valid && rad) ? __ldg(A.F.s + (int64_t)T * nc + cell) : 0.f;
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
  int wi0 = 0, wj0 = 0;
  uint64_t ovr = 0, inwin = 0;
  if (mode == MODE_WINDOW) {
    int ci, cj;
    float rdummy;
    move_sample(P, F, cs, sn, u1, v1, x1, y1, late, ci, cj, rdummy);
    wi0 = min(max(ci - kWin / 2, 0), g - W);
    wj0 = min(max(cj - kWin / 2, 0), g - W);
    for (int li = 0; li < W; ++li) {
      for (int lj = 0; lj < W; ++lj) {
        int i2 = wi0 + li, j2 = wj0 + lj;
        int lb = li * kWin + lj;
        int di = i2 - i1 + P.del, dj = j2 - j1 + P.del;
        if (di >= 0 && di < P.m && dj >= 0 && dj < P.m) inwin |= 1ull << lb;
        if (through_obstacle(P, A.F.mask, T, i1, j1, i2, j2)) ovr |= 1ull << lb;
      }
    }
  }
#pragma unroll
  for (int w = 0; w < kWinWords; ++w) win[w * nthr + tid] = 0u;

  float sumR = 0.f;
  uint32_t n_drop = 0, n_misbin = 0;
  uint32_t* dense = nullptr;
  const int mm = P.m * P.m;

  // ---- realisations in chunks ---------------------------------------------
  for (int base = 0; base < P.nrzns; base += A.rc) {
    const int clen = min(A.rc, P.nrzns - base);
    __syncthreads();  // modes staged / previous chunk consumed
    for (int q = a; q < clen; q += nwarps) {
      const float* y = A.F.Y + ((int64_t)T * P.nrzns + base + q) * nm;
      float sum_x = 0;
      float sum_y = 0;
      for (int k = 0; k < nm; k++) sum_x += modes[k * 32 + lane] * __ldg(y + k);
      for (int k = 0; k < nm; k++) sum_y += modes[(nm + k) * 32 + lane] * __ldg(y + k);
      // extract_velocity, src/build_model.cu:389-401: mean + sum over modes
      vel[q * 32 + lane] = make_float2(u1 + sum_x, v1 + sum_y);
    }
    __syncthreads();
    if (mode == MODE_FIXED) {
      for (int q = 0; q < clen; ++q) sumR += r_fixed;
    } else if (mode != MODE_LOST) {
      for (int q = 0; q < clen; ++q) {
        const float2 vv = vel[q * 32 + lane];
        int i2, j2;
        float r;
        move_sample(P, F, cs, sn, vv.x, vv.y, x1, y1, late, i2, j2, r);
        float rad2 = 0.f;
        if (rad) rad2 = __ldg(A.F.s + (int64_t)(T + 1) * nc + (int64_t)i2 * g + j2);
        float r_step = step_reward(P, F, rad1, rad2);
        r += r_step;
        const unsigned li = (unsigned)(i2 - wi0), lj = (unsigned)(j2 - wj0);
        if (mode == MODE_WINDOW && li < (unsigned)W && lj < (unsigned)W) {
          const int lb = (int)li * kWin + (int)lj;
          if ((ovr >> lb) & 1ull) r = P.r_out;
          if ((inwin >> lb) & 1ull) {
            win[(lb >> 1) * nthr + tid] += 1u << ((lb & 1) << 4);
          } else {
            n_drop++;
            int di = i2 - i1 + P.del, dj = j2 - j1 + P.del;
            if (di < P.m && dj < P.m) n_misbin++;
          }
        } else {
          if (through_obstacle(P, A.F.mask, T, i1, j1, i2, j2)) r = P.r_out;
          const int di = i2 - i1 + P.del, dj = j2 - j1 + P.del;
          if (di >= 0 && di < P.m && dj >= 0 && dj < P.m) {
            if (mode == MODE_WINDOW) {
              // switch this row to a dense m*m histogram from the pool
              unsigned long long slot = atomicAdd(A.counters + CTR_POOL, 1ull);
              atomicAdd(A.counters + CTR_OVERFLOW_ROWS, 1ull);
              if (slot < (unsigned long long)A.pool_units) {
                dense = A.pool + slot * (unsigned long long)mm;
                for (int b = 0; b < mm; ++b) dense[b] = 0u;
                for (int lb = 0; lb < W * kWin; ++lb) {
                  if ((lb % kWin) >= W) continue;
                  uint32_t c = (win[(lb >> 1) * nthr + tid] >> ((lb & 1) << 4)) & 0xFFFFu;
                  if (c) {
                    int ii = wi0 + lb / kWin - i1 + P.del, jj = wj0 + lb % kWin - j1 + P.del;
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
        }
        sumR += r;
        if (mode == MODE_LOST) break;
      }
    }
  }
  if (n_drop) atomicAdd(A.counters + CTR_DROPPED, (unsigned long long)n_drop);
  if (n_misbin) atomicAdd(A.counters + CTR_MISBIN, (unsigned long long)n_misbin);
  if (mode == MODE_LOST) atomicOr(reinterpret_cast<unsigned int*>(A.counters + CTR_FLAGS), FLAG_POOL_EXHAUSTED);

  // ---- row lengths, tile scan, emission ------------------------------------
  int nnz = 0;
  if (valid) {
    if (mode == MODE_FIXED) {
      nnz = 1;
    } else if (mode == MODE_WINDOW) {
#pragma unroll
      for (int w = 0; w < kWinWords; ++w) {
        uint32_t word = win[w * nthr + tid];
        nnz += ((word & 0xFFFFu) != 0u) + ((word >> 16) != 0u);
      }
    } else if (mode == MODE_DENSE) {
      for (int b = 0; b < mm; ++b) nnz += dense[b] != 0u;
    }
  }
  const int lrow = lane * P.na + a;  // row order inside the tile: cell-major, then action
  __syncthreads();
  scan[lrow] = nnz;
  __syncthreads();
  // exclusive scan over scan[0..nthr) in place
  int v = scan[tid];
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t2 = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t2;
  }
  if (lane == 31) warp_tot[a] = incl;
  __syncthreads();
  if (a == 0) {
    int wt = lane < nwarps ? warp_tot[lane] : 0;
    int wi = wt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int t2 = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t2;
    }
    if (lane < nwarps) warp_tot[lane] = wi - wt;  // exclusive warp offsets
    if (lane == 31) {
      // wi on lane 31 is the tile total
      tile_base_sh = atomicAdd(A.counters + CTR_STAGE, (unsigned long long)wi);
      const int64_t tile = (int64_t)T * A.tiles_per_layer + blockIdx.x;
      A.tile_base[tile] = (int64_t)tile_base_sh;
      A.tile_len[tile] = wi;
    }
  }
  __syncthreads();
  scan[tid] = warp_tot[a] + incl - v;
  __syncthreads();
  if (!valid) return;
  const int excl = scan[lrow];
  const int64_t grow = ((int64_t)T * nc + cell) * P.na + a;
  A.row_off[grow] = (uint32_t)excl;
  A.R[grow] = sumR / P.nrzns;  // compute_mean, src/build_model.cu:567
  const unsigned long long tb = tile_base_sh;
  if (mode == MODE_LOST) return;
  unsigned long long off = tb + (unsigned long long)excl;
  if (off + (unsigned long long)nnz > (unsigned long long)A.stage_cap) return;  // host re-runs
  CntT* scnt = reinterpret_cast<CntT*>(A.stage_cnt);
  const int64_t next_layer = (int64_t)(T + 1) * nc;
  if (mode == MODE_FIXED) {
    A.stage_col[off] = (int32_t)(next_layer + cell);
    scnt[off] = (CntT)P.nrzns;
  } else if (mode == MODE_WINDOW) {
    for (int lb = 0; lb < W * kWin; ++lb) {
      uint32_t c = (win[(lb >> 1) * nthr + tid] >> ((lb & 1) << 4)) & 0xFFFFu;
      if (c) {
        int i2 = wi0 + lb / kWin, j2 = wj0 + lb % kWin;
        A.stage_col[off] = (int32_t)(next_layer + (int64_t)i2 * g + j2);
        scnt[off] = (CntT)c;
        ++off;
      }
    }
  } else {  // MODE_DENSE: bins in reference order
    for (int b = 0; b < mm; ++b) {
      uint32_t c = dense[b];
      if (c) {
        int i2 = b / P.m + i1 - P.del, j2 = b % P.m + j1 - P.del;
        A.stage_col[off] = (int32_t)(next_layer + (int64_t)i2 * g + j2);
        scnt[off] = (CntT)c;
        ++off;
      }
    }
  }
}

// K2: exclusive scan of the tile lengths (tile order == row order) with one
// CTA; each thread owns a contiguous run of tiles.
__global__ void k_scan_tiles(const int32_t* __restrict__ tile_len, int64_t n_tiles,
                             int64_t* __restrict__ canon, int64_t* __restrict__ total) {
  __shared__ int64_t part[1024];
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int64_t per = (n_tiles + nthr - 1) / nthr;
  const int64_t b = min((int64_t)tid * per, n_tiles), e = min(b + per, n_tiles);
  int64_t s = 0;
  for (int64_t i = b; i < e; ++i) s += tile_len[i];
  part[tid] = s;
  __syncthreads();
  if (tid == 0) {
    int64_t run = 0;
    for (int k = 0; k < nthr; ++k) {
      int64_t x = part[k];
      part[k] = run;
      run += x;
    }
    *total = run;
  }
  __syncthreads();
  int64_t run = part[tid];
  for (int64_t i = b; i < e; ++i) {
    canon[i] = run;
    run += tile_len[i];
  }
}

// K3: one CTA per tile: move the tile's entries from staging to their
// canonical position and write row_ptr for the tile's rows.
template <typename CntT, typename PtrT>
__global__ void k_assemble(AssembleArgs A) {
  const int64_t tile = blockIdx.x;
  const int64_t src = A.tile_base[tile];
  const int64_t dst = A.canon[tile];
  const int len = A.tile_len[tile];
  const int32_t* __restrict__ scol = A.stage_col + src;
  const CntT* __restrict__ scnt = reinterpret_cast<const CntT*>(A.stage_cnt) + src;
  int32_t* __restrict__ dcol = A.col + dst;
  CntT* __restrict__ dcnt = reinterpret_cast<CntT*>(A.cnt) + dst;
  for (int k = threadIdx.x; k < len; k += blockDim.x) {
    dcol[k] = scol[k];
    dcnt[k] = scnt[k];
  }
  const int64_t layer = tile / A.tiles_per_layer;
  const int64_t tl = tile - layer * A.tiles_per_layer;
  const int64_t cb = tl * 32;
  const int64_t ce = min(cb + 32, A.ncells);
  const int64_t r0 = (layer * A.ncells + cb) * A.na;
  const int64_t r1 = (layer * A.ncells + ce) * A.na;
  PtrT* rp = reinterpret_cast<PtrT*>(A.row_ptr);
  for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) rp[r] = (PtrT)(dst + A.row_off[r]);
  if (tile == A.n_tiles - 1 && threadIdx.x == 0) rp[A.n_rows] = (PtrT)A.total_nnz;
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

size_t build_smem_bytes(int na, int nm, int rc) {
  return (size_t)rc * 32 * sizeof(float2) + (size_t)2 * nm * 32 * sizeof(float) +
         (size_t)kWinWords * 32 * na * sizeof(uint32_t) + (size_t)32 * na * sizeof(int);
}

cudaError_t launch_build_tiles(const BuildArgs& A, int count_bits, int n_layers,
                               cudaStream_t st) {
  dim3 grid((unsigned)A.tiles_per_layer, (unsigned)n_layers);
  dim3 block((unsigned)(32 * A.P.na));
  size_t sm = build_smem_bytes(A.P.na, A.P.nm, A.rc);
  cudaError_t e;
  if (count_bits == 16) {
    e = cudaFuncSetAttribute(k_build_tiles<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
    if (e != cudaSuccess) return e;
    k_build_tiles<uint16_t><<<grid, block, sm, st>>>(A);
  } else {
    e = cudaFuncSetAttribute(k_build_tiles<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sm);
    if (e != cudaSuccess) return e;
    k_build_tiles<uint32_t><<<grid, block, sm, st>>>(A);
  }
  return cudaGetLastError();
}

cudaError_t launch_scan_tiles(const int32_t* tile_len, int64_t n_tiles, int64_t* canon,
                              int64_t* total, cudaStream_t st) {
  k_scan_tiles<<<1, 1024, 0, st>>>(tile_len, n_tiles, canon, total);
  return cudaGetLastError();
}

cudaError_t launch_assemble(const AssembleArgs& A, int count_bits, int index_bits,
                            cudaStream_t st) {
  dim3 grid((unsigned)A.n_tiles), block(256);
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
