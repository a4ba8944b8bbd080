// K7: policy rollout evaluation.
//
// The reference evaluates a solved policy in Python, one realisation after
// another (Post_processing/plot_e2eGPU_policy.py:433-474, the loop of
// plot_exact_trajectory_set_DP without policy interpolation): from the start
// cell it follows the policy, moving with Grid.move_exact
// (Post_processing/grid_world.py:160-271) on continuous positions, until the
// target, an edge or obstacle cell, or the last time step; get_metrics
// (:776-797) summarises success rate, travel time and energies.
//
// Here one thread follows one realisation.  The arithmetic is the reference's
// under NumPy's float32 scalar rules (a Python number with a float32 stays
// float32): every multiply, add, divide is a separately rounded float32
// operation (__fmul_rn / __fadd_rn / __fdiv_rn, never contracted), the cell
// index is NumPy's float32 floor division and remainder, headings' cosines are
// the float32 roundings of the double cosines of round(i*2pi/n, 14).  The one
// chosen order is the velocity dot product u + sum_k ui_k * Y_k: a sequential
// fma chain over the modes (the reference's np.matmul leaves that order to
// its BLAS library).
//
// With interp set, the actions after the first are interpolated from the
// policy of the four cells around the vehicle's position (the script's
// with_policy_interp branch: get_interpolated_action :174-198,
// interpolate_action_angles :111-171, bilinear / triangle interpolation
// :37-108) in the types NumPy gives them: the bilinear form in float32 with
// its two small matrix products as separately rounded products summed in
// order (NumPy's float32 matmul of these shapes, checked on the host), the
// triangle form (next to the target cell) with float64 weights, after which
// the reference's position is float64 and this kernel's movement continues in
// double.  Heading atan2, its cosine and the speed's square root are CUDA's;
// the reference takes them from the host libm and NumPy's scalar power, which
// can differ in the last bit, so interpolated trajectories agree with the
// reference's per realisation almost always rather than bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.h"

#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)

namespace e2e {
namespace {

struct RolloutArgs {
  DevFields F;
  const int32_t* policy;
  const float* xs;     // g, the reference's Python grid ticks (float32)
  const float* ys;
  const float* speed;  // na
  const float* cosv;   // na
  const float* sinv;   // na
  int g, nt, nm, na, tsg, it, jt, i0, j0, nrzns, nrzns_field;
  int interp;          // actions after the first interpolated from the policy
  float dt, dj, di;
  int8_t* success;     // per realisation: 1 target, 0 failed, -1 undecided, -2 invalid policy entry
  int32_t* ttime;
  float* energy;       // 3 per realisation: sum F^2, sum mean scalar field, their difference
  int32_t* final_tij;  // 3 per realisation
};

// NumPy's float32 divmod (fmod, exact correction of the quotient, floor with
// the 0.5 guard); returns floor(a / b) and sets rem.
__device__ __forceinline__ float divmod32(float a, float b, float& rem) {
  float mod = fmodf(a, b);
  float div = __fdiv_rn(__fsub_rn(a, mod), b);
  if (mod != 0.f) {
    if ((b < 0.f) != (mod < 0.f)) {
      mod = __fadd_rn(mod, b);
      div = __fsub_rn(div, 1.0f);
    }
  } else {
    mod = copysignf(0.f, b);
  }
  float fl;
  if (div != 0.f) {
    fl = floorf(div);
    if (__fsub_rn(div, fl) > 0.5f) fl = __fadd_rn(fl, 1.0f);
  } else {
    fl = copysignf(0.f, __fdiv_rn(a, b));
  }
  rem = mod;
  return fl;
}

// NumPy's float64 divmod (the same algorithm as divmod32, in double)
__device__ __forceinline__ double divmod64(double a, double b, double& rem) {
  double mod = fmod(a, b);
  double div = (a - mod) / b;
  if (mod != 0.0) {
    if ((b < 0.0) != (mod < 0.0)) {
      mod += b;
      div -= 1.0;
    }
  } else {
    mod = copysign(0.0, b);
  }
  double fl;
  if (div != 0.0) {
    fl = floor(div);
    if (div - fl > 0.5) fl += 1.0;
  } else {
    fl = copysign(0.0, a / b);
  }
  rem = mod;
  return fl;
}

// Python's float % with a positive modulus (CPython float_rem)
__device__ __forceinline__ double py_mod(double a, double b) {
  double m = fmod(a, b);
  if (m != 0.0) {
    if ((b < 0.0) != (m < 0.0)) m += b;
  } else {
    m = copysign(0.0, b);
  }
  return m;
}

// The interpolated action at (x, y) in cell (t, i, j): speed (float32, or
// double in *speed_d with *wide_out set when the triangle form ran or the
// position was already double) and heading in [0, 2pi).
struct Interp {
  float speed;
  double speed_d, angle;
  bool wide;
  bool bad;  // a support cell's policy entry is not an action (the reference's lookup fails there)
};

__device__ Interp interp_action(const RolloutArgs& A, int t, int i, int j, float xf, float yf, double xd, double yd,
                                bool wide) {
  const int g = A.g;
  const int64_t nc = (int64_t)g * g;
  const double x = wide ? xd : (double)xf, y = wide ? yd : (double)yf;
  const int fx = (x - (double)A.xs[j] < 0.0) ? -1 : 1;  // f(delx), the sign of an exact difference
  const int fy = (y - (double)A.ys[g - 1 - i] < 0.0) ? -1 : 1;
  const int si[4] = {i, i - fy, i, i - fy}, sj[4] = {j, j, j + fx, j + fx};
  int term[4];
  float vx[4], vy[4];
  Interp r;
  r.bad = false;
  for (int k = 0; k < 4; ++k) {
    term[k] = (si[k] == A.it && sj[k] == A.jt) ? 1 : 0;
    const int a = A.policy[(int64_t)t * nc + (int64_t)si[k] * g + sj[k]];
    if (a < 0 || a >= A.na) r.bad = true;
    const int aa = r.bad ? 0 : a;
    vx[k] = __fmul_rn(A.speed[aa], A.cosv[aa]);
    vy[k] = __fmul_rn(A.speed[aa], A.sinv[aa]);
  }
  bool tri = false;
  if (term[0] == 0 && term[1] == 0 && term[2] == 1) {  // [0,0,1,1] / [0,0,1,0]
    vx[2] = vx[0];
    vx[3] = vx[1];
    vy[2] = vy[0];
    vy[3] = vy[1];
  } else if (term[0] == 0 && term[1] == 1 && term[2] == 0) {  // [0,1,0,1] / [0,1,0,0]
    vx[1] = vx[0];
    vx[3] = vx[2];
    vy[1] = vy[0];
    vy[3] = vy[2];
  } else if (term[0] == 0 && term[1] == 0 && term[2] == 0 && term[3] == 1) {
    tri = true;
  }
  const float x1 = A.xs[j], x2 = A.xs[j + fx];
  const float y1 = A.ys[g - 1 - i], y2 = A.ys[g - 1 - (i - fy)];
  double ivx, ivy;
  if (!tri && !wide) {  // float32: denom * (x_vec @ (val_mat @ y_vec))
    const float den = __fdiv_rn(1.0f, __fmul_rn(__fsub_rn(x2, x1), __fsub_rn(y2, y1)));
    const float xa = __fsub_rn(x2, xf), xb = __fsub_rn(xf, x1);
    const float ya = __fsub_rn(y2, yf), yb = __fsub_rn(yf, y1);
    auto bil = [&](const float* v) {
      const float in0 = __fadd_rn(__fmul_rn(v[0], ya), __fmul_rn(v[1], yb));
      const float in1 = __fadd_rn(__fmul_rn(v[2], ya), __fmul_rn(v[3], yb));
      return __fmul_rn(den, __fadd_rn(__fmul_rn(xa, in0), __fmul_rn(xb, in1)));
    };
    const float fvx = bil(vx), fvy = bil(vy);
    r.angle = py_mod(atan2((double)fvy, (double)fvx) + 2.0 * M_PI, 2.0 * M_PI);
    r.speed = sqrtf(__fadd_rn(__fmul_rn(fvx, fvx), __fmul_rn(fvy, fvy)));
    r.speed_d = r.speed;
    r.wide = false;
    return r;
  }
  if (!tri) {  // position already double: the same form promoted to float64
    const double den = (double)__fdiv_rn(1.0f, __fmul_rn(__fsub_rn(x2, x1), __fsub_rn(y2, y1)));
    const double xa = (double)x2 - x, xb = x - (double)x1, ya = (double)y2 - y, yb = y - (double)y1;
    auto bil = [&](const float* v) {
      const double in0 = __dadd_rn(__dmul_rn(v[0], ya), __dmul_rn(v[1], yb));
      const double in1 = __dadd_rn(__dmul_rn(v[2], ya), __dmul_rn(v[3], yb));
      return __dmul_rn(den, __dadd_rn(__dmul_rn(xa, in0), __dmul_rn(xb, in1)));
    };
    ivx = bil(vx);
    ivy = bil(vy);
  } else {  // triangle through (x1, y1), (x1, y2), (x2, y1); weights float32 (double once wide), then float64
    const float d23y = __fsub_rn(y2, y1), d13x = __fsub_rn(x1, x2), d32x = __fsub_rn(x2, x1);
    const float d0y = __fsub_rn(y1, y1);  // b1 - b3 and b3 - b1 of the reference's expressions
    const double den = __fadd_rn(__fmul_rn(d23y, d13x), __fmul_rn(d32x, d0y));
    double w0, w1;
    if (!wide) {
      const float xa3 = __fsub_rn(xf, x2), yb3 = __fsub_rn(yf, y1);
      w0 = __fadd_rn(__fmul_rn(d23y, xa3), __fmul_rn(d32x, yb3));
      w1 = __fadd_rn(__fmul_rn(d0y, xa3), __fmul_rn(d13x, yb3));
    } else {
      const double xa3 = x - (double)x2, yb3 = y - (double)y1;
      w0 = __dadd_rn(__dmul_rn(d23y, xa3), __dmul_rn(d32x, yb3));
      w1 = __dadd_rn(__dmul_rn(d0y, xa3), __dmul_rn(d13x, yb3));
    }
    w0 = w0 / den;
    w1 = w1 / den;
    const double w2 = (1.0 - w0) - w1;
    ivx = __dadd_rn(__dadd_rn(__dmul_rn(vx[0], w0), __dmul_rn(vx[1], w1)), __dmul_rn(vx[2], w2));
    ivy = __dadd_rn(__dadd_rn(__dmul_rn(vy[0], w0), __dmul_rn(vy[1], w1)), __dmul_rn(vy[2], w2));
  }
  r.angle = py_mod(atan2(ivy, ivx) + 2.0 * M_PI, 2.0 * M_PI);
  r.speed_d = sqrt(__dadd_rn(__dmul_rn(ivx, ivx), __dmul_rn(ivy, ivy)));
  r.speed = (float)r.speed_d;
  r.wide = true;
  return r;
}

__global__ void __launch_bounds__(128) k_rollout(RolloutArgs A) {
  const int rzn = blockIdx.x * blockDim.x + threadIdx.x;
  if (rzn >= A.nrzns) return;
  const int g = A.g, nt = A.nt, nm = A.nm;
  const int64_t nc = (int64_t)g * g;
  auto term = [&](int i, int j) { return i >= A.it && i < A.it + A.tsg && j >= A.jt && j < A.jt + A.tsg; };
  int t = 0, i = A.i0, j = A.j0;
  float x = A.xs[j], y = A.ys[g - 1 - i];
  double xd = 0.0, yd = 0.0;  // the position once it is float64 (after a triangle-form action)
  bool wide = false;
  // the action: speed and heading cosine / sine (float32), or in double for a
  // float64 interpolated action
  bool act_d = false;
  float thr = 0.f, cth = 0.f, sth = 0.f;
  double thr_d = 0.0, cth_d = 0.0, sth_d = 0.0;
  const float xs0 = A.xs[0], xsn = A.xs[g - 1], ys0 = A.ys[0], ysn = A.ys[g - 1];
  int a = A.policy[(int64_t)t * nc + (int64_t)i * g + j];
  if (a >= 0 && a < A.na) {
    thr = A.speed[a];
    cth = A.cosv[a];
    sth = A.sinv[a];
  }
  int success = -1;  // -1: undecided (the reference's None)
  float e_cons = 0.f, e_col = 0.f, e_net = 0.f;
  int travel = 0;
  for (int it = 0; it < nt; ++it) {
    if (success == -1) {
      if (!act_d && (a < 0 || a >= A.na)) {  // the reference indexes its action list with it and fails
        success = -2;
        break;
      }
      const int64_t cell = (int64_t)t * nc + (int64_t)i * g + j;
      float dx_ = 0.f, dy_ = 0.f;
      const float* yk = A.F.Y + ((int64_t)t * A.nrzns_field + rzn) * nm;
      for (int k = 0; k < nm; ++k) {
        const float w = yk[k];
        dx_ = fmaf(A.F.ui[((int64_t)t * nm + k) * nc + (int64_t)i * g + j], w, dx_);
        dy_ = fmaf(A.F.vi[((int64_t)t * nm + k) * nc + (int64_t)i * g + j], w, dy_);
      }
      const float vx = __fadd_rn(A.F.u[cell], dx_);
      const float vy = __fadd_rn(A.F.v[cell], dy_);
      const float rad1 = A.F.s[cell];
      if (!term(i, j) && t < nt - 1 && !act_d) {  // move_exact
        const float thrust = thr;
        const float vnx = __fadd_rn(__fmul_rn(thrust, cth), vx);
        const float vny = __fadd_rn(__fmul_rn(thrust, sth), vy);
        float xn = __fadd_rn(x, __fmul_rn(vnx, A.dt));
        float yn = __fadd_rn(y, __fmul_rn(vny, A.dt));
        if (xn > xsn) xn = xsn;
        else if (xn < xs0) xn = xs0;
        if (yn > ysn) yn = ysn;
        else if (yn < ys0) yn = ys0;
        x = xn;
        y = yn;
        float remx, remy;
        float xind = divmod32(__fsub_rn(xn, xs0), A.dj, remx);
        float yind = divmod32(-__fsub_rn(yn, ysn), A.di, remy);
        if (remx >= __fmul_rn(0.5f, A.dj)) xind = __fadd_rn(xind, 1.0f);
        if (remy >= __fmul_rn(0.5f, A.di)) yind = __fadd_rn(yind, 1.0f);
        if (!(isnan(xind) || isnan(yind))) {
          i = (int)yind;
          j = (int)xind;
        }
        t += 1;
      } else if (!term(i, j) && t < nt - 1) {  // move_exact with a float64 action: the position becomes float64
        const double vnx = __dadd_rn(__dmul_rn(thr_d, cth_d), (double)vx);
        const double vny = __dadd_rn(__dmul_rn(thr_d, sth_d), (double)vy);
        double xn = __dadd_rn(wide ? xd : (double)x, __dmul_rn(vnx, (double)A.dt));
        double yn = __dadd_rn(wide ? yd : (double)y, __dmul_rn(vny, (double)A.dt));
        if (xn > xsn) xn = xsn;
        else if (xn < xs0) xn = xs0;
        if (yn > ysn) yn = ysn;
        else if (yn < ys0) yn = ys0;
        xd = xn;
        yd = yn;
        x = (float)xn;
        y = (float)yn;
        wide = true;
        double remx, remy;
        double xind = divmod64(xn - (double)xs0, (double)A.dj, remx);
        double yind = divmod64(-(yn - (double)ysn), (double)A.di, remy);
        if (remx >= (double)__fmul_rn(0.5f, A.dj)) xind += 1.0;
        if (remy >= (double)__fmul_rn(0.5f, A.di)) yind += 1.0;
        if (!(isnan(xind) || isnan(yind))) {
          i = (int)yind;
          j = (int)xind;
        }
        t += 1;
      }
      const float rad2 = A.F.s[(int64_t)t * nc + (int64_t)i * g + j];
      travel += 1;
      const float sp = act_d ? (float)thr_d : thr;
      const float sp2 = __fmul_rn(sp, sp);
      const float half = __fdiv_rn(__fadd_rn(rad2, rad1), 2.0f);
      e_cons = __fadd_rn(e_cons, sp2);
      e_col = __fadd_rn(e_col, half);
      e_net = __fadd_rn(e_net, __fsub_rn(sp2, half));
    }
    if (i == 0 || i == g - 1 || j == 0 || j == g - 1 || A.F.mask[(int64_t)t * nc + (int64_t)i * g + j] == 1)
      success = 0;
    if (!term(i, j) && t < nt - 1 && success == -1) {
      if (A.interp) {
        const Interp r = interp_action(A, t, i, j, x, y, xd, yd, wide);
        if (r.bad) {
          success = -2;
          break;
        }
        act_d = r.wide;
        thr = r.speed;
        thr_d = r.speed_d;
        cth = (float)cos(r.angle);
        sth = (float)sin(r.angle);
        cth_d = cos(r.angle);
        sth_d = sin(r.angle);
      } else {
        a = A.policy[(int64_t)t * nc + (int64_t)i * g + j];
        if (a >= 0 && a < A.na) {
          thr = A.speed[a];
          cth = A.cosv[a];
          sth = A.sinv[a];
        }
      }
    }
    else if (term(i, j)) success = 1;
    else success = 0;
  }
  A.success[rzn] = (int8_t)success;
  A.ttime[rzn] = travel;
  A.energy[3 * rzn] = e_cons;
  A.energy[3 * rzn + 1] = e_col;
  A.energy[3 * rzn + 2] = e_net;
  A.final_tij[3 * rzn] = t;
  A.final_tij[3 * rzn + 1] = i;
  A.final_tij[3 * rzn + 2] = j;
}

// round(x, 14) of Python: the correctly rounded 14-decimal string, read back
double round14(double x) {
  char buf[64];
  std::snprintf(buf, sizeof(buf), "%.14f", x);
  return std::strtod(buf, nullptr);
}

}  // namespace
}  // namespace e2e

extern "C" e2e_status e2e_rollout(const e2e_problem* p, const e2e_fields* f, int fields_where,
                                  const int32_t* policy, int policy_where, const e2e_rollout_opts* opts,
                                  int8_t* success_out, int32_t* time_out, float* energy_out,
                                  int32_t* final_out, e2e_rollout_stats* stats, void* stream) {
  using namespace e2e;
  e2e_status vs = validate_problem(p);
  if (vs != E2E_OK) return vs;
  if (!f || !policy || !opts) return fail(E2E_ERR_INVALID, "null argument");
  if ((fields_where != E2E_HOST && fields_where != E2E_DEVICE) ||
      (policy_where != E2E_HOST && policy_where != E2E_DEVICE))
    return fail(E2E_ERR_INVALID, "bad memory location");
  const int g = p->gsize;
  if (opts->i_start < 0 || opts->i_start >= g || opts->j_start < 0 || opts->j_start >= g)
    return fail(E2E_ERR_INVALID, "start cell outside the grid");
  const int n = opts->n_rzns > 0 ? std::min(opts->n_rzns, p->nrzns) : p->nrzns;
  cudaStream_t st = (cudaStream_t)stream;
  DeviceScratch scratch(st);
  FieldsOnDevice fd;
  e2e_status s = fields_to_device(p, f, fields_where, st, &fd, &scratch);
  if (s != E2E_OK) return s;
  const int64_t ns = (int64_t)g * g * p->nt;
  const int32_t* dpol = policy;
  if (policy_where == E2E_HOST) {
    int32_t* d = nullptr;
    CK(dalloc((void**)&d, sizeof(int32_t) * ns, st));
    scratch.add(d);
    CK(cudaMemcpyAsync(d, policy, sizeof(int32_t) * ns, cudaMemcpyHostToDevice, st));
    dpol = d;
  }
  // the reference's Python grid and action set, in its scalar types
  const int na = p->num_actions, nsp = p->num_ac_speeds, nan_ = p->num_ac_angles;
  std::vector<float> tab(2 * (size_t)g + 3 * (size_t)na);
  const float dx = p->dx, dy = p->dy;
  for (int k = 0; k < g; ++k) {
    tab[k] = (dx / 2.0f) + ((float)k * dx);
    tab[g + k] = (dy / 2.0f) + ((float)k * dy);
  }
  std::vector<float> speeds;
  if (nsp == 1) {
    speeds.push_back(p->F);
  } else {
    const float dF = p->F / (float)nsp;
    for (int k = 0; k < nsp; ++k) speeds.push_back((float)(k + 1) * dF);
  }
  for (int sIdx = 0; sIdx < nsp; ++sIdx)
    for (int aIdx = 0; aIdx < nan_; ++aIdx) {
      const int q = sIdx * nan_ + aIdx;
      const double ang = round14((double)(aIdx * 2) * M_PI / (double)nan_);
      tab[2 * g + q] = speeds[sIdx];
      tab[2 * g + na + q] = (float)std::cos(ang);
      tab[2 * g + 2 * na + q] = (float)std::sin(ang);
    }
  float* dtab = nullptr;
  CK(dalloc((void**)&dtab, sizeof(float) * tab.size(), st));
  scratch.add(dtab);
  CK(cudaMemcpyAsync(dtab, tab.data(), sizeof(float) * tab.size(), cudaMemcpyHostToDevice, st));
  int8_t* d_succ = nullptr;
  int32_t *d_time = nullptr, *d_fin = nullptr;
  float* d_en = nullptr;
  CK(dalloc((void**)&d_succ, (size_t)n + 16, st));
  scratch.add(d_succ);
  CK(dalloc((void**)&d_time, sizeof(int32_t) * n, st));
  scratch.add(d_time);
  CK(dalloc((void**)&d_fin, sizeof(int32_t) * 3 * n, st));
  scratch.add(d_fin);
  CK(dalloc((void**)&d_en, sizeof(float) * 3 * n, st));
  scratch.add(d_en);
  RolloutArgs A;
  A.F = fd.F;
  A.policy = dpol;
  A.xs = dtab;
  A.ys = dtab + g;
  A.speed = dtab + 2 * g;
  A.cosv = dtab + 2 * g + na;
  A.sinv = dtab + 2 * g + 2 * na;
  A.g = g;
  A.nt = p->nt;
  A.nm = p->nmodes;
  A.na = na;
  A.tsg = p->term_subgrid_size;
  A.it = p->i_term;
  A.jt = p->j_term;
  A.i0 = opts->i_start;
  A.j0 = opts->j_start;
  A.nrzns = n;
  A.nrzns_field = p->nrzns;
  A.dt = p->dt;
  A.interp = (opts->flags & E2E_ROLLOUT_INTERP) ? 1 : 0;
  A.dj = std::fabs(tab[1] - tab[0]);
  A.di = std::fabs(tab[g + 1] - tab[g]);
  A.success = d_succ;
  A.ttime = d_time;
  A.energy = d_en;
  A.final_tij = d_fin;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, st));
  k_rollout<<<(n + 127) / 128, 128, 0, st>>>(A);
  CK(cudaGetLastError());
  CK(cudaEventRecord(e1, st));
  std::vector<int8_t> hs((size_t)n);
  std::vector<int32_t> ht((size_t)n);
  std::vector<float> he(3 * (size_t)n);
  CK(cudaMemcpyAsync(hs.data(), d_succ, (size_t)n, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(ht.data(), d_time, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(he.data(), d_en, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, st));
  if (final_out) CK(cudaMemcpyAsync(final_out, d_fin, sizeof(int32_t) * 3 * n, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (success_out) std::memcpy(success_out, hs.data(), (size_t)n);
  if (time_out) std::memcpy(time_out, ht.data(), sizeof(int32_t) * n);
  if (energy_out) std::memcpy(energy_out, he.data(), sizeof(float) * 3 * n);
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->n = n;
    double st_[4] = {0, 0, 0, 0};
    for (int k = 0; k < n; ++k) {
      if (hs[k] == 1) {
        stats->successes++;
        st_[0] += ht[k];
        st_[1] += he[3 * k];
        st_[2] += he[3 * k + 1];
        st_[3] += he[3 * k + 2];
      } else if (hs[k] == 0) {
        stats->failures++;
      } else if (hs[k] == -1) {
        stats->undecided++;
      } else {
        stats->invalid++;
      }
    }
    stats->success_rate = n ? (double)stats->successes / n : 0.0;
    const double ns_ = stats->successes ? (double)stats->successes : 1.0;
    stats->mean_time = st_[0] / ns_;
    stats->mean_energy_cons = st_[1] / ns_;
    stats->mean_energy_col = st_[2] / ns_;
    stats->mean_net_energy = st_[3] / ns_;
    stats->seconds = ms * 1e-3;
  }
  return E2E_OK;
}
