// Which cells a builder CTA takes: the order of a layer's warp groups.
// Host and device code (the builder kernel and a CPU test of the mapping).
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define E2E_TILE_ORDER_FN __host__ __device__ __forceinline__
#else
#define E2E_TILE_ORDER_FN inline
#endif

namespace e2e {

// Which group of a layer's cells a builder warp takes.  A warp holds cpw
// consecutive cells (cpw = 32 / warps per CTA); its group index is also its
// emission tile, so the canonical CSR order does not depend on which CTA ran
// it.  Warps whose windows can reach the grid's edge run the slower counting
// loop with the domain clamps; mixed into a CTA of plain warps they keep the
// plain warps waiting at every chunk barrier.  So the slots of a layer list
// the groups with a cell within kEdgeBand cells of the border first, then the
// interior groups, each in index order, and CTA `tile` takes slots
// tile * nwarps ... + nwarps - 1.  Identity when cpw does not divide g or the
// grid has no interior.
static constexpr int kEdgeBand = 7;  // window reach (kWin / 2 + 1) plus a mean-flow drift of two cells

E2E_TILE_ORDER_FN int64_t group_of_slot(int64_t s, int g, int cpw) {
  const int64_t gq = g / cpw, ngroups = (int64_t)g * gq;
  const int qlo = (kEdgeBand + cpw - 1) / cpw, qhi = (g - kEdgeBand) / cpw - 1;
  const int ni = qhi - qlo + 1, nri = g - 2 * kEdgeBand;
  if (g % cpw != 0 || ni <= 0 || nri <= 0 || s >= ngroups) return s;
  const int64_t ne_row = gq - ni, top = (int64_t)kEdgeBand * gq, mid = (int64_t)nri * ne_row;
  const int64_t n_edge = 2 * top + mid;
  if (s >= n_edge) {  // interior: rows [E, g-E), groups [qlo, qhi]
    const int64_t k = s - n_edge;
    return (kEdgeBand + k / ni) * gq + qlo + k % ni;
  }
  if (s < top) return s;  // rows [0, E)
  int64_t e = s - top;
  if (e < mid) {  // the edge groups of an interior row: [0, qlo) and (qhi, gq)
    const int64_t k = e % ne_row;
    return (kEdgeBand + e / ne_row) * gq + (k < qlo ? k : k + ni);
  }
  return (int64_t)(g - kEdgeBand) * gq + (e - mid);  // rows [g-E, g)
}

}  // namespace e2e
