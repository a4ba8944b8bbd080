// Shared device definitions: problem constants, the per-sample motion /
// reward model and the obstacle test of the Monte-Carlo transition builder.
//
// Per-sample arithmetic is written with the same C expressions, in the same
// order, as the reference's device functions (src/build_model.cu:231-477), so
// that nvcc makes the same floating-point contraction decisions and the next
// cell of every sample is bit-identical to the reference's.  Do not rewrite
// these expressions "equivalently": a*b+c and c+a*b may contract differently.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace e2e {

// Problem constants in the form the kernels use (prob_params slots,
// src/build_model.cu:1032-1055, plus the derived grid ticks).
struct DevProblem {
  int g;            // gsize
  int nt;
  int nm;           // nmodes
  int nrzns;
  int na;           // num_actions
  int m;            // neighb_gsize
  int del;          // (m-1)/2
  int it, jt, tsg;  // terminal subgrid
  int reward_type;
  int unit_step;    // Dj == 1 && Di == 1: snapping by rint (exactly remainderf's result)
  float dt, r_out, r_term, alpha;
  float xs0, xsn, ys0, ysn;  // xs[0], xs[g-1], ys[0], ys[g-1]
  float Dj, Di;              // fabsf(xs[1]-xs[0]), fabsf(ys[1]-ys[0])
  float axmax, aymax;        // xsn - xs0 and -(ys0 - ysn): snapping-coordinate bounds
  const float* xs;           // device, g
  const float* ys;           // device, g
  const float* ac_speed;     // device, na
  const float* ac_cos;       // device, na: cosf(angle) evaluated on the device
  const float* ac_sin;       // device, na
};

struct DevFields {
  const float* u;
  const float* v;
  const float* ui;
  const float* vi;
  const float* Y;
  const float* s;
  const int32_t* mask;
};

// calculate_one_step_reward, src/build_model.cu:231-265 (same expressions).
__device__ __forceinline__ float step_reward(const DevProblem& P, float ac_speed, float rad1,
                                             float rad2) {
  int method = P.reward_type;
  float alpha = P.alpha;
  float Cr = 1;
  float Cf = 1;
  float Ct = 0.01;
  float dt = P.dt;
  float energy_reward, time_reward;
  if (method == 0) return -dt;
  else if (method == 1) {
    return -(Cf * ac_speed * ac_speed + Ct) * dt;
  } else if (method == 2) {
    return ((Cr * (rad2 + rad1) / 2) - (Cf * ac_speed * ac_speed) - Ct) * dt;
  } else if (method == 3) {
    return ((Cr * (rad2 + rad1) / 2) - Ct) * dt;
  } else if (method == 4) {
    energy_reward = -(ac_speed * ac_speed) * dt;
    time_reward = -dt;
    return alpha * energy_reward + (1 - alpha) * time_reward;
  } else
    return 0;
}

// Advection of move(), src/build_model.cu:284-289: the reference's expressions.
__device__ __forceinline__ void advect(const DevProblem& P, float F, float cs, float sn, float vx,
                                      float vy, float x, float y, float& xnew, float& ynew) {
  float vnetx = F * cs + vx;
  float vnety = F * sn + vy;
  xnew = x + (vnetx * P.dt);
  ynew = y + (vnety * P.dt);
}

// Snapping of move(), src/build_model.cu:313-335: nearest cell centre with
// ties rounded up.  UNIT (Dj == Di == 1): remainderf(a, 1) == a - rintf(a)
// exactly and (a - rem)/1 == rintf(a), so rintf gives the same indices.
template <bool UNIT>
__device__ __forceinline__ void snap(const DevProblem& P, float xnew, float ynew, int32_t& xind,
                                     int32_t& yind) {
  if (UNIT) {
    float ax = xnew - P.xs0;
    float ay = -(ynew - P.ysn);
    float nx = rintf(ax);
    float ny = rintf(ay);
    float remx = ax - nx;
    float remy = ay - ny;
    xind = (int32_t)nx + (remx >= 0.5f ? 1 : 0);
    yind = (int32_t)ny + (remy >= 0.5f ? 1 : 0);
  } else {
    float remx = remainderf((xnew - P.xs0), P.Dj);
    float remy = remainderf(-(ynew - P.ysn), P.Di);
    xind = ((xnew - P.xs0) - remx) / P.Dj;
    yind = (-(ynew - P.ysn) - remy) / P.Di;
    if (remx >= 0.5 * P.Dj) xind += 1;
    if (remy >= 0.5 * P.Di) yind += 1;
  }
}

// move(), src/build_model.cu:268-356: advect one step, clamp to the domain,
// snap to the nearest cell centre, add edge / terminal / late-time rewards.
// (x, y) is the centre of the start cell; on return (i2, j2) is the next cell.
template <bool UNIT>
__device__ __forceinline__ void move_sample(const DevProblem& P, float F, float cs, float sn,
                                            float vx, float vy, float x, float y, bool late,
                                            int& i2, int& j2, float& r) {
  float xnew, ynew;
  advect(P, F, cs, sn, vx, vy, x, y, xnew, ynew);
  r = 0;
  if (xnew > P.xsn) {
    xnew = P.xsn;
    r += P.r_out;
  } else if (xnew < P.xs0) {
    xnew = P.xs0;
    r += P.r_out;
  }
  if (ynew > P.ysn) {
    ynew = P.ysn;
    r += P.r_out;
  } else if (ynew < P.ys0) {
    ynew = P.ys0;
    r += P.r_out;
  }
  int32_t xind, yind;
  snap<UNIT>(P, xnew, ynew, xind, yind);
  i2 = yind;
  j2 = xind;
  int32_t n = P.g - 1;
  if (i2 == 0 || i2 == n || j2 == 0 || j2 == n) r += P.r_out;
  if ((i2 >= P.it && i2 < P.it + P.tsg) && (j2 >= P.jt && j2 < P.jt + P.tsg)) {
    r += P.r_term;
  } else {
    if (late) r += 0.05 * P.r_out;
  }
}

// The landing cell of move_sample without the rewards, for unit cell spacing.
//
// The clamps of move() are applied to the snapping coordinates instead:
// ax = xnew - xs0 clamped to [0, xsn - xs0] and ay = -(ynew - ysn) clamped to
// [0, -(ys0 - ysn)].  Rounding is monotone, so inside the domain the values
// are the reference's, beyond an edge they equal the reference's clamped
// values, and a NaN becomes 0 (fmaxf returns the non-NaN operand), which is
// the index the reference's float-to-int conversion gives a NaN.
//
// Index: the reference takes n = rint(a) (remainderf with spacing 1) and adds
// 1 when a - n >= 0.5, i.e. it rounds half up: index = floor(a + 0.5), exactly.
// With round-toward-minus-infinity adds, w = RD(a + 0.5) has floor(w) ==
// floor(a + 0.5) (integers below 2^24 are floats, so w cannot drop below it),
// and RD(w + 1.5*2^23) == 1.5*2^23 + floor(w) because floats in [2^23, 2^24)
// are spaced by 1; the integer is then the low mantissa bits.
__device__ __forceinline__ int32_t round_half_up_index(float a, int32_t bias) {
  const float w = __fadd_rd(a, 0.5f);
  const float t = __fadd_rd(w, 12582912.0f);  // 1.5 * 2^23
  return __float_as_int(t) - bias;            // bias = bits of 1.5*2^23 (+ window origin)
}

// advect() on (x, y) pairs with the packed float2 instructions of sm_100:
// each component is the same fused multiply-add, rounded the same way.
__device__ __forceinline__ float2 advect2(float2 FF, float2 csn, float2 v, float2 dt2, float2 xy) {
  const float2 vnet = __ffma2_rn(FF, csn, v);  // (F*cs + vx, F*sn + vy)
  return __ffma2_rn(vnet, dt2, xy);            // (x + vnetx*dt, y + vnety*dt)
}

// round_half_up_index() of both coordinates with the packed adds.
__device__ __forceinline__ void round_half_up_index2(float2 a, int32_t bias_x, int32_t bias_y,
                                                     int32_t& jx, int32_t& iy) {
  const float2 w = __fadd2_rd(a, make_float2(0.5f, 0.5f));
  const float2 t = __fadd2_rd(w, make_float2(12582912.0f, 12582912.0f));
  jx = __float_as_int(t.x) - bias_x;
  iy = __float_as_int(t.y) - bias_y;
}

__device__ __forceinline__ void land_unit(const DevProblem& P, float F, float cs, float sn,
                                          float vx, float vy, float x, float y, int& i2, int& j2) {
  float xnew, ynew;
  advect(P, F, cs, sn, vx, vy, x, y, xnew, ynew);
  const float ax = fminf(fmaxf(xnew - P.xs0, 0.0f), P.axmax);
  const float ay = fminf(fmaxf(-(ynew - P.ysn), 0.0f), P.aymax);
  j2 = round_half_up_index(ax, 0x4B400000);
  i2 = round_half_up_index(ay, 0x4B400000);
}

// General spacing: the reference's clamps (if / else) and remainderf snap.
__device__ __forceinline__ void land_general(const DevProblem& P, float F, float cs, float sn,
                                             float vx, float vy, float x, float y, int& i2, int& j2) {
  float xnew, ynew;
  advect(P, F, cs, sn, vx, vy, x, y, xnew, ynew);
  if (xnew > P.xsn) xnew = P.xsn;
  else if (xnew < P.xs0) xnew = P.xs0;
  if (ynew > P.ysn) ynew = P.ysn;
  else if (ynew < P.ys0) ynew = P.ys0;
  int32_t xind, yind;
  snap<false>(P, xnew, ynew, xind, yind);
  i2 = yind;
  j2 = xind;
}

template <bool UNIT>
__device__ __forceinline__ void land(const DevProblem& P, float F, float cs, float sn, float vx,
                                     float vy, float x, float y, int& i2, int& j2) {
  if (UNIT) land_unit(P, F, cs, sn, vx, vy, x, y, i2, j2);
  else land_general(P, F, cs, sn, vx, vy, x, y, i2, j2);
}

__device__ __forceinline__ bool is_terminal(const DevProblem& P, int i, int j) {
  return (i >= P.it && i < P.it + P.tsg) && (j >= P.jt && j < P.jt + P.tsg);
}

// is_within_band, src/build_model.cu:419-441 (same expressions).
__device__ __forceinline__ bool within_band(const DevProblem& P, int i, int j, int i1, int j1,
                                            int i2, int j2) {
  if (i1 == i2 || j1 == j2) return true;
  float cell_diag = fabsf(P.xs[1] - P.xs[0]) * 1.414213;
  float x = P.xs[j], y = P.ys[P.g - 1 - i];
  float x1 = P.xs[j1], y1 = P.ys[P.g - 1 - i1];
  float x2 = P.xs[j2], y2 = P.ys[P.g - 1 - i2];
  float A = (y2 - y1) / (x2 - x1);
  float B = -1;
  float C = y1 - (A * x1);
  float dist_btw_pt_line = fabsf(A * x + B * y + C) / sqrtf((A * A) + (B * B));
  return dist_btw_pt_line < cell_diag;
}

// goes_through_obstacle, src/build_model.cu:444-477: any obstacle cell (at T
// or T+1, mask value 1) in the bounding box of S1 -> S2, other than S1, that
// lies within the band of the S1-S2 segment.
__device__ __forceinline__ bool through_obstacle(const DevProblem& P, const int32_t* mask,
                                                 int T, int i1, int j1, int i2, int j2) {
  const int64_t nc = (int64_t)P.g * P.g;
  const int32_t* m0 = mask + (int64_t)T * nc;
  const int32_t* m1 = m0 + nc;
  int imin = min(i1, i2), imax = max(i1, i2);
  int jmin = min(j1, j2), jmax = max(j1, j2);
  for (int i = imin; i <= imax; i++) {
    for (int j = jmin; j <= jmax; j++) {
      if (!(i == i1 && j == j1)) {
        int64_t sp = (int64_t)j + (int64_t)P.g * i;
        if (__ldg(m0 + sp) == 1 || __ldg(m1 + sp) == 1) {
          if (within_band(P, i, j, i1, j1, i2, j2)) return true;
        }
      }
    }
  }
  return false;
}

// Value of one model row: R + (sum of count * V[col]) / nrzns, the sum taken
// in entry (ascending next-state) order with fused multiply-adds.  Every
// solver path of this package evaluates rows through this function, so a
// state gets bit-identical values from the Jacobi, layered, batched and
// served solvers.
__device__ __forceinline__ float finish_row(float R, float acc, float inv_scale_unused,
                                            int nrzns, bool counts) {
  return counts ? R + acc / (float)nrzns : R + acc;
}

__device__ __forceinline__ float to_f(uint16_t c) { return (float)c; }
__device__ __forceinline__ float to_f(uint32_t c) { return (float)c; }
__device__ __forceinline__ float to_f(float c) { return c; }

}  // namespace e2e
