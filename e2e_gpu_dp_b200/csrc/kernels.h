// Internal interface between the host orchestration (capi.cu, batch.cu,
// server.cpp) and the CUDA kernels.  Not part of the public C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace e2e {

// slots of the builder's device counter block (unsigned long long each)
enum : int {
  CTR_STAGE = 0,          // staging entries allocated (== nnz when it fits)
  CTR_DROPPED = 1,        // samples outside the m x m neighbourhood
  CTR_MISBIN = 2,         // ... of which the reference would file under a wrong bin
  CTR_OVERFLOW_ROWS = 3,  // rows that left the fast window
  CTR_POOL = 4,           // dense-histogram pool slots requested
  CTR_FLAGS = 5,          // error flags
  CTR_NEXT_TILE = 6,      // fused build+backup: the next tile to take
  CTR_COUNT = 8
};
// FLAG_WAIT_TIMEOUT: a wait of the fused build+backup for the next layer's
// completion ran out of its bound (the pass's values are not valid)
enum : unsigned int { FLAG_POOL_EXHAUSTED = 1u, FLAG_WAIT_TIMEOUT = 2u };

struct BuildArgs {
  DevProblem P;
  DevFields F;
  int t0;               // first layer of this launch (blockIdx.y offset)
  int tiles_per_layer;  // CTAs per layer = ceil(ncells / 32); emission tiles are warps
  int rc;               // realisations per warp-private velocity chunk
  int ybufs;            // chunk coefficient buffers in shared memory: 1, or 2 (one CTA barrier a chunk)
  int lanes_log2;       // lanes per cell = 1 << lanes_log2 >= na
  int32_t* stage_col;
  void* stage_cnt;
  int64_t stage_cap;
  unsigned long long* counters;  // CTR_COUNT slots
  uint32_t* row_off;             // per row: offset inside its tile
  int64_t* tile_base;            // per tile: staging offset
  int32_t* tile_len;             // per tile: entries
  float* R;                      // per row (state-major, Ns * na)
  float* sumR;                   // nullable: per-row reward sums (before the division)
  uint32_t* pool;                // pool_units x m*m dense histograms
  int64_t pool_units;
  float* V;                      // fused build+backup: values (ns), layer t+1 read, layer t written
  int32_t* pi;                   // fused build+backup: policy (ns)
  unsigned int* layer_done;      // fused build+backup: per (layer, grid row), cells backed up (nt x g, zeroed per pass)
  unsigned long long wait_ns;    // fused build+backup: bound of a wait for a layer's completion
  unsigned int wait_extra;       // test hook: raises the waits' targets so that none completes
};

struct AssembleArgs {
  int64_t n_tiles, tiles_per_layer, cells_per_tile, ncells, n_rows, total_nnz;
  int na;
  const int64_t* tile_base;
  const int32_t* tile_len;
  const int64_t* canon;
  const uint32_t* row_off;
  const int32_t* stage_col;
  const void* stage_cnt;
  void* row_ptr;
  int32_t* col;
  void* cnt;
};

int build_lanes_log2(int na);
size_t build_smem_bytes(int na, int nm, int rc, bool unit, int ybufs);
// builder CTAs that fit one SM with this dynamic shared memory (the lowest of
// the staging kernels, 16- and 32-bit counts, and the fused kernel), from the
// kernels' registers and static shared memory and the device's limits
int build_ctas_per_sm(int na, size_t smem, bool unit);
cudaError_t launch_build_tiles(const BuildArgs& A, int count_bits, int n_layers, cudaStream_t st);
// The fused build+backup of every layer (uses A.V, A.pi, A.pool, A.counters,
// A.layer_done; no staging): one cooperative launch whose CTAs take the tiles
// of layers nt-2 down to 0 in order and back each row up as soon as layer t+1
// is complete.  *grid receives the CTAs launched.
cudaError_t launch_build_fused(const BuildArgs& A, cudaStream_t st, int* grid);
cudaError_t launch_scan_tiles(const int32_t* tile_len, int64_t n_tiles, int64_t* canon,
                              int64_t* total, int64_t* block_sums, cudaStream_t st);
cudaError_t launch_assemble(const AssembleArgs& A, int count_bits, int index_bits,
                            cudaStream_t st);
cudaError_t launch_action_trig(const float* angle, int n, float* cosv, float* sinv,
                               cudaStream_t st);

// ---- value iteration ----------------------------------------------------------
enum : int { CNT_U16 = 0, CNT_U32 = 1, VAL_F32 = 2 };

struct ViModel {
  int64_t ns, n_row_states;
  int na, nrzns;
  int count_type;   // CNT_U16 / CNT_U32 / VAL_F32
  int index_bits;   // 32 / 64
  const void* row_ptr;
  const int32_t* col;
  const void* cnt;
  const float* R;
};

// One sweep over states [s_begin, s_end): Vout[s] = max_a Q(s, a), pi[s] = argmax.
// resid (nullable): FP64 max |Vout - Vin| accumulated with atomicMax on the bits.
cudaError_t launch_vi_sweep(const ViModel& M, int64_t s_begin, int64_t s_end, const float* Vin,
                            float* Vout, int32_t* pi, unsigned long long* resid, cudaStream_t st);
cudaError_t launch_vi_sweep_f64(const ViModel& M, int64_t s_begin, int64_t s_end, double* V,
                                cudaStream_t st);
// max |V - Vd| into err[0], max |Vd| into err[1] (bits of non-negative doubles)
cudaError_t launch_compare_f64(const float* V, const double* Vd, int64_t n,
                               unsigned long long* err, cudaStream_t st);

// ---- sliced copy of a model for value iteration (vi_pack.cu) ------------------
// entry layouts of the sliced copy
enum : int {
  ENT_PACKED = 0,  // uint32 per entry: 16-bit window offset | uint16 count << 16
  ENT_OFF16 = 1,   // uint16 window offset + uint32 count / float value arrays
  ENT_I32 = 2      // int32 column + count array (models without window geometry)
};

struct ViPack {
  int64_t ns, nc;          // states; states per layer (ns when the model has no layers)
  int64_t cpl, nchunks;    // chunks of 32 states per layer; all chunks
  int64_t n_row_states;    // states that own rows
  int64_t slot_rows;       // slot rows of 32 entries
  int nlayers, na, na_pad, nrzns, count_type, ent_mode;
  int g, del;              // grid side and window half-width (window-offset column base)
  const int64_t* chunk_slot;  // nchunks + 1: first slot row of each chunk
  const uint16_t* maxlen;     // nchunks * na_pad: slot rows per (chunk, action)
  const void* col;            // slot_rows * 32: packed entries, uint16 offsets or int32 columns
  const void* cnt;            // slot_rows * 32: counts / values (null for ENT_PACKED)
  const float* R;             // nchunks * na * 32: [chunk][action][lane]
};

struct PackStore {
  ViPack v{};
  void* bufs[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int64_t bytes = 0;
};

// Build the sliced copy of a state-major CSR model.  nc = states per layer
// (0: none); g, del = grid side and window half-width of a layered model built
// on a g x g grid (0: unknown, int32 columns).
cudaError_t build_pack(const ViModel& M, int64_t nc, int g, int del, PackStore* out, cudaStream_t st);
void free_pack(PackStore* p);
// bytes one sweep over the pack moves (entries with padding, R, tables, V)
int64_t pack_sweep_bytes(const ViPack& P);
// tune bits of the sweeps: L2 bulk prefetch of the chunk a warp takes next
// (the next layer's, when layered) and/or of the chunk it starts; the lean
// kernel (no entry look-ahead, 8 CTAs per SM) instead of the look-ahead one;
// for the Jacobi sweep of the packed layout, the TMA-staged kernel
enum : int { VI_TUNE_PF_NEXT = 1, VI_TUNE_PF_CURRENT = 2, VI_TUNE_LEAN = 4, VI_TUNE_TMA = 8 };
// One Jacobi sweep over chunks [c_begin, c_end).
// err: device word for bounded-wait failures (needed by the TMA-staged kernel)
cudaError_t launch_vi_chunks(const ViPack& P, int64_t c_begin, int64_t c_end, const float* Vin,
                             float* Vout, int32_t* pi, unsigned long long* resid, cudaStream_t st,
                             int tune, unsigned int* err = nullptr);
// The whole layered schedule in one cooperative launch, in place on V.
// sync: two zeroed words (barrier count, error bits); groups: warps per chunk
// (1, 2, 4, 8; 0 picks one).
cudaError_t launch_vi_layered(const ViPack& P, float* V, int32_t* pi, unsigned int* sync, int groups,
                              cudaStream_t st, int tune);


// ---- many models in one persistent launch (batched and served solves) ----------
// A job is one model's layered solve: V and policy outputs, and optionally a
// re-targeted copy of R for the cells around a target (served requests).
struct ViJob {
  ViPack P;
  float* V;
  int32_t* pi;
  const float* Rwin;     // null, or R of cells [wi0, wi0+wh) x [wj0, wj0+ww):
                         // [layer < nlayers-1][wh][ww][na]
  int ti, tj, tsg;       // terminal subgrid of the target (when Rwin is set)
  int wi0, wj0, wh, ww;
};
struct ViBatchHeader {
  int njobs, max_layers, pad0, pad1;
};
// Device table: header | jobs[job_cap] | cum[job_cap + 1] | nact[layer_cap].
// Jobs sorted by nlayers, descending; cum = prefix sums of their chunks per
// layer; nact[k] = jobs with more than k layers.  Step k of the launch works
// on layer nlayers-1-k of jobs [0, nact[k]): chunk items [0, cum[nact[k]]),
// each waiting only for its own job's next layer.
size_t vi_batch_table_bytes(int job_cap, int layer_cap);
constexpr int kViBatchJobCap = 1024;  // jobs of one batched launch at most
constexpr size_t kViBatchJobsOffset = 64;  // header padded to 64 bytes
// CTAs of the batch kernel that fit on the device at once
int vi_batch_capacity(int ent_mode, int count_type, int tune);
// done: zeroed [job_cap][layer_cap] completion counters; err: zeroed error word;
// grid <= vi_batch_capacity (co-resident CTAs)
cudaError_t launch_vi_batch(const void* table, int job_cap, int layer_cap, int ent_mode, int count_type,
                            int groups, int grid, int tune, int* done, unsigned int* err, cudaStream_t st);

}  // namespace e2e
