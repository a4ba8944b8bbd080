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
  CTR_COUNT = 8
};
enum : unsigned int { FLAG_POOL_EXHAUSTED = 1u };

struct BuildArgs {
  DevProblem P;
  DevFields F;
  int t0;               // first layer of this launch (blockIdx.y offset)
  int tiles_per_layer;  // CTAs per layer = ceil(ncells / 32); emission tiles are warps
  int rc;               // (unused) realisations per chunk
  int lanes_log2;       // lanes per cell = 1 << lanes_log2 >= na
  int32_t* stage_col;
  void* stage_cnt;
  int64_t stage_cap;
  unsigned long long* counters;  // CTR_COUNT slots
  uint32_t* row_off;             // per row: offset inside its tile
  int64_t* tile_base;            // per tile: staging offset
  int32_t* tile_len;             // per tile: entries
  float* R;                      // per row (state-major, Ns * na)
  uint32_t* pool;                // pool_units x m*m dense histograms
  int64_t pool_units;
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
size_t build_smem_bytes(int na, int nm, int rc);
cudaError_t launch_build_tiles(const BuildArgs& A, int count_bits, int n_layers, cudaStream_t st);
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

}  // namespace e2e
