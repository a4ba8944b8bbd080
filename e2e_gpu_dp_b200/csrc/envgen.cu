// Environment generator on the GPU: double-gyre realisations -> per-time
// rank reduction -> interpolation to the planning grid, plus the moving
// scalar "cloud" field and the obstacle mask
// (src/data_input/build_environment_DG_with_westward_clouds.py:106-590).
//
// Per time step t (one at a time, so memory is one step's matrices):
//   k_env_realisations  vx, vy, phi of every (sample k, coarse cell) in double,
//                       the reference's expressions in its evaluation order
//                       without contraction (:130-147, 20-84 for the cloud)
//   k_env_center        column means in sample order (np.mean over axis 1 is a
//                       sequential sum for this layout) and the centred matrix
//   rank reduction      the leading n_modes singular triplets of the centred
//                       matrix by a randomized range finder (n_modes + 10
//                       columns from a fixed hash, two power iterations) in
//                       hand-written double kernels: products X B and X^T B,
//                       Gram-Schmidt twice for the orthonormal bases, and the
//                       SVD of the projected matrix through its QR factor and a
//                       one-sided Jacobi SVD of that factor (relative accuracy,
//                       like LAPACK's).  Accepted when the explicit residual
//                       |X - Q Q^T X|_F is below 1e-10 s_1 (then every kept
//                       singular value is exact to ~|R|^2/s_k), or when s_1 is
//                       below 1e-10 of the data's own size (the t = 0 matrices,
//                       rounding noise of the centring, whose vectors no
//                       implementation determines); otherwise re-run with twice
//                       the columns and four power iterations.  The first
//                       n_modes give coefficients u_k s_k and modes v_k, signs
//                       fixed so that each coefficient column's largest-magnitude
//                       entry is positive (the reference's np.linalg.svd leaves
//                       the sign to LAPACK)
// then, for all steps, k_env_interpolate: the reference's griddata 'linear' on
// the coarse cell centres, evaluated from a table of (triangle vertices,
// barycentric weights) per fine point that the caller builds from the same
// Delaunay triangulation (scipy's), summed in griddata's order in double
// without contraction; points outside the hull read 0 (np.nan_to_num of the
// fill value).
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "e2e_dp.h"
#include "internal.h"

using namespace e2e;

#define CK(call)                                        \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(_e, #call); \
  } while (0)
namespace {

constexpr double kPi = 3.141592653589793;  // math.pi

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

struct RealArgs {
  int g, nws, t;
  double tt;  // ts[t] = t * dt
  double dxy, A, eps, wlo, whi, wx, wy;
  double* Xv;  // nws x 2n: vx then vy
  double* Xp;  // nws x n: phi
};

// DG_velocity_field.vx_vy / phi / sample_w / get_ij_from_xy (:130-166)
__global__ void k_env_realisations(RealArgs a) {
  const int n = a.g * a.g;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)a.nws * n) return;
  const int k = (int)(idx / n), c = (int)(idx - (int64_t)k * n);
  const int i = c / a.g, j = c - i * a.g;
  // w = w_i + r (w_f - w_i), r = k / (n_wsamples - 1)
  const double r = a.nws > 1 ? (double)k / (double)(a.nws - 1) : 0.0;
  const double w = add(a.wlo, mul(r, sub(a.whi, a.wlo)));
  const double x = mul(add(0.5, (double)j), a.dxy);
  const double y = mul(add(0.5, (double)(a.g - 1 - i)), a.dxy);
  const double swt = sin(mul(w, a.tt));
  // f = eps sin(wt) x^2 + (1 - 2 eps sin(wt)) x;  fx = 2 eps sin(wt) (x - 1) + 1
  const double term1 = mul(mul(a.eps, swt), mul(x, x));
  const double e2s = mul(mul(2.0, a.eps), swt);
  const double term2 = mul(sub(1.0, e2s), x);
  const double f = add(term1, term2);
  const double fx = add(mul(e2s, sub(x, 1.0)), 1.0);
  const double swf = sin(mul(a.wx, f)), cwf = cos(mul(a.wx, f));
  const double swy = sin(mul(a.wy, y)), cwy = cos(mul(a.wy, y));
  const double vx = -mul(mul(mul(mul(0.5, a.A), kPi), swf), cwy);
  const double vy = mul(mul(mul(mul(a.A, kPi), swy), fx), cwf);
  const double ph = mul(mul(a.A, sin(mul(kPi, f))), swy);
  a.Xv[(int64_t)k * 2 * n + c] = vx;
  a.Xv[(int64_t)k * 2 * n + n + c] = vy;
  a.Xp[(int64_t)k * n + c] = ph;
}

// column means (sequential sum over samples, then / n_wsamples) and centring
__global__ void k_env_center(double* X, int nws, int ncols, double* mean) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncols) return;
  double s = X[c];
  for (int k = 1; k < nws; ++k) s = add(s, X[(int64_t)k * ncols + c]);
  const double m = __ddiv_rn(s, (double)nws);
  mean[c] = m;
  for (int k = 0; k < nws; ++k) X[(int64_t)k * ncols + c] = sub(X[(int64_t)k * ncols + c], m);
}

// From the SVD of the centred matrix X (nws x ncols): coefficients C (nws x r)
// and modes M (r x ncols), mode q = the q-th largest singular value:
// C[k][q] = Us[k + q ldu] s_q (the left singular vectors scaled, rank_reduction's
// u1 diag(s1)), M[q][c] = Vs[c + q ldv] (Vh's rows).  Signs: the
// largest-magnitude coefficient of each mode is made positive.
struct ModeArgs {
  int nws, ncols, r;
  const double* S;   // singular values, descending
  const double* Us;  // left singular vectors (sample side), column q at Us + q * ldu
  int ldu;
  const double* Vs;  // right singular vectors (grid side), column q at Vs + q * ldv
  int ldv;
  double* C;         // nws x r
  double* M;         // r x ncols
  double* svals;     // r
};

__global__ void k_env_modes(ModeArgs a) {
  const int q = blockIdx.x;  // one block per mode
  const double s = a.S[q];
  __shared__ double best_v[32];
  __shared__ int best_k[32];
  const double* u = a.Us + (int64_t)q * a.ldu;
  double bv = -1.0;
  int bk = 0x7fffffff;
  for (int k = threadIdx.x; k < a.nws; k += blockDim.x) {
    const double v = fabs(u[k] * s);
    if (v > bv || (v == bv && k < bk)) {
      bv = v;
      bk = k;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
    const int ok = __shfl_xor_sync(0xffffffffu, bk, o);
    if (ov > bv || (ov == bv && ok < bk)) {
      bv = ov;
      bk = ok;
    }
  }
  if ((threadIdx.x & 31) == 0) {
    best_v[threadIdx.x >> 5] = bv;
    best_k[threadIdx.x >> 5] = bk;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (best_v[w] > bv || (best_v[w] == bv && best_k[w] < bk)) {
        bv = best_v[w];
        bk = best_k[w];
      }
    best_k[0] = bk;
  }
  __syncthreads();
  const double sgn = u[best_k[0]] < 0.0 ? -1.0 : 1.0;
  if (threadIdx.x == 0) a.svals[q] = s;
  for (int k = threadIdx.x; k < a.nws; k += blockDim.x) a.C[(int64_t)k * a.r + q] = sgn * (u[k] * s);
  const double* v = a.Vs + (int64_t)q * a.ldv;
  for (int c = threadIdx.x; c < a.ncols; c += blockDim.x) a.M[(int64_t)q * a.ncols + c] = sgn * v[c];
}

// test matrix of the range finder: deterministic values in [-1, 1) from a
// 64-bit mix of the index (any matrix of full rank with the range works)
__global__ void k_env_test_matrix(double* O, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint64_t z = (uint64_t)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  O[i] = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// coarse arrays of step t: [u, v, phi, ui_0.., vi_0.., phi_i_0..] (3 + 3r arrays
// of n) and the coefficients of both rank reductions.  The reference holds the
// coarse means and modes in float32 arrays except all_phi_mat, a float64 array
// (:271), so every value but phi's mean is rounded to float before it is
// interpolated.
__global__ void k_env_store(int n, int nws, int r, const double* mv, const double* mp, const double* Mv,
                            const double* Mp, const double* Cv, const double* Cp, double* coarse, float* yi,
                            float* phi_yi) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nb = (int64_t)(3 + 3 * r) * n;
  if (idx < nb) {
    const int b = (int)(idx / n), c = (int)(idx - (int64_t)b * n);
    double v;
    if (b == 0) v = mv[c];
    else if (b == 1) v = mv[n + c];
    else if (b == 2) v = mp[c];
    else if (b < 3 + r) v = Mv[(int64_t)(b - 3) * 2 * n + c];
    else if (b < 3 + 2 * r) v = Mv[(int64_t)(b - 3 - r) * 2 * n + n + c];
    else v = Mp[(int64_t)(b - 3 - 2 * r) * n + c];
    coarse[idx] = b == 2 ? v : (double)(float)v;
  }
  const int64_t nc = (int64_t)nws * r;
  if (idx < nc) {
    yi[idx] = (float)Cv[idx];
    phi_yi[idx] = (float)Cp[idx];
  }
}

struct InterpArgs {
  int nt, r, n, G2;
  const double* coarse;  // nt x (3 + 3r) x n
  const int32_t* vert;   // G2 x 3 (vert[0] < 0: outside the hull)
  const double* wgt;     // G2 x 3
  unsigned int* err;     // set when a vertex index is outside the coarse grid
  float *u, *v, *phi, *ui, *vi, *phi_i;
};

// LinearNDInterpolator's evaluation (scipy/interpolate/_interpnd.pyx
// _do_evaluate): out = 0; out += c_j * value[vertex_j] for j = 0..2 in double
__global__ void k_env_interpolate(InterpArgs a) {
  const int nb = 3 + 3 * a.r;
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)a.nt * nb * a.G2) return;
  const int p = (int)(idx % a.G2);
  const int64_t tb = idx / a.G2;
  const int b = (int)(tb % nb), t = (int)(tb / nb);
  const double* src = a.coarse + ((int64_t)t * nb + b) * a.n;
  float out = 0.f;  // np.nan_to_num of the fill value outside the hull
  const int v0 = a.vert[3 * p], v1 = a.vert[3 * p + 1], v2 = a.vert[3 * p + 2];
  if (v0 >= 0) {
    if (v0 >= a.n || v1 < 0 || v1 >= a.n || v2 < 0 || v2 >= a.n) {
      atomicOr(a.err, 1u);  // a caller's table that does not index the coarse grid
    } else {
      double o = 0.0;
      o = add(o, mul(a.wgt[3 * p + 0], src[v0]));
      o = add(o, mul(a.wgt[3 * p + 1], src[v1]));
      o = add(o, mul(a.wgt[3 * p + 2], src[v2]));
      out = isnan(o) ? 0.f : (float)o;
    }
  }
  float* dst;
  if (b == 0) dst = a.u + (int64_t)t * a.G2;
  else if (b == 1) dst = a.v + (int64_t)t * a.G2;
  else if (b == 2) dst = a.phi + (int64_t)t * a.G2;
  else if (b < 3 + a.r) dst = a.ui + ((int64_t)t * a.r + (b - 3)) * a.G2;
  else if (b < 3 + 2 * a.r) dst = a.vi + ((int64_t)t * a.r + (b - 3 - a.r)) * a.G2;
  else dst = a.phi_i + ((int64_t)t * a.r + (b - 3 - 2 * a.r)) * a.G2;
  dst[p] = out;
}

// DG_scalar_field.generate_phi (:20-98) on the fine grid (its interpolate_degree
// is the default 1, so T = t / 2), and fill_obstacles (:441-468)
struct CloudArgs {
  int nt, G;
  double dxy;  // fine spacing
  double A_sc;
  int obst_mode;
  double ou, ol, ow, osx, osy;
  float* s;
  int32_t* mask;
};

__global__ void k_env_cloud(CloudArgs a) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t G2 = (int64_t)a.G * a.G;
  if (idx >= (int64_t)a.nt * G2) return;
  const int t = (int)(idx / G2);
  const int p = (int)(idx - (int64_t)t * G2);
  const int i = p / a.G, j = p - i * a.G;
  const double x = mul(add(0.5, (double)j), a.dxy);
  const double xl = mul(add(0.5, (double)(a.G - 1)), a.dxy);  // xs[-1]
  const double T = __ddiv_rn((double)t, 2.0);
  const double l = __ddiv_rn(xl, 2.0);
  const double dom = add(xl, a.dxy);
  const double xt = add(x, mul(T, a.dxy));
  double f;
  if (xt <= l) {
    f = 1.0;
  } else if (l < xt && xt < add(l, mul(0.2, dom))) {
    const double slope = __ddiv_rn(1.0, mul(-0.2, dom));
    f = add(1.0, mul(slope, sub(x, sub(l, mul(T, a.dxy)))));
  } else {
    f = 0.0;
  }
  a.s[idx] = (float)mul(a.A_sc, f);
  int m = 0;
  if (a.obst_mode == E2E_OBST_STATIC) {
    const int ru = (int)(0.4 * a.G), rd = (int)(0.5 * a.G), cl = (int)(0.5 * a.G), cr = (int)(0.6 * a.G);
    m = (i >= ru && i < rd && j >= cl && j < cr) ? 1 : 0;
  } else if (a.obst_mode == E2E_OBST_DYNAMIC) {
    const double clf = floor(add(a.ol, mul((double)t, a.osx)));
    const double ruf = floor(add(a.ou, mul((double)t, a.osy)));
    const double crf = trunc(add(clf, a.ow)), rdf = trunc(add(ruf, a.ow));
    const double hi = (double)(a.G - 1);
    const bool inside = (0.0 < clf && clf < hi) && (0.0 < crf && crf < hi) && (0.0 < ruf && ruf < hi) &&
                        (0.0 < rdf && rdf < hi);
    m = (inside && i >= (int)ruf && i < (int)rdf && j >= (int)clf && j < (int)crf) ? 1 : 0;
  }
  a.mask[idx] = m;
}

// ---- rank reduction: the leading singular triplets of the centred matrix ----
//
// X is row-major nws x ncols on the device.  A randomized range finder with k
// columns (n_modes + 10): Q = orth(X Om), two power iterations
// Q <- orth(X orth(X^T Q)), Bt = X^T Q (ncols x k), the explicit residual
// |X - Q Bt^T|_F, then the SVD of Bt through its QR: Bt = Qb R, R = U_R S V_R^T
// by one-sided Jacobi (relative accuracy: each singular value of R equals one
// of Bt's to about eps s_1, so a Gram-matrix eigensolve's (s_1/s_k)^2 loss is
// avoided), Ub = Qb U_R, and the sample-side vectors L = Q V_R.  Every product
// and reduction runs in a fixed order (warp trees, segment sums in segment
// order), so a generation is deterministic.  Matrices besides X are
// column-major with the leading dimension of their row count.

constexpr int kRrMaxK = 64;       // range-finder columns at most
constexpr int kRrMaxSweeps = 60;  // Jacobi sweeps at most (convergence is quadratic)

// partial products of X^T B over row segments: P[seg][c][j] = sum over the
// segment's rows i, in order, of X[i][j] B[i][c]; a thread per column j
template <int K>
__global__ void __launch_bounds__(128) k_rr_xtb(const double* X, int nws, int ncols, const double* B, int ldb,
                                                int k, int seg_rows, double* P) {
  __shared__ double Bs[32][K];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = blockIdx.y * seg_rows, i1 = min(nws, i0 + seg_rows);
  double acc[K];
#pragma unroll
  for (int c = 0; c < K; ++c) acc[c] = 0.0;
  for (int it = i0; it < i1; it += 32) {
    const int nrow = min(32, i1 - it);
    __syncthreads();
    for (int e = threadIdx.x; e < 32 * K; e += blockDim.x) {
      const int rr = e / K, c = e - rr * K;
      Bs[rr][c] = (rr < nrow && c < k) ? B[(int64_t)c * ldb + it + rr] : 0.0;
    }
    __syncthreads();
    if (j < ncols) {
      for (int rr = 0; rr < nrow; ++rr) {
        const double x = X[(int64_t)(it + rr) * ncols + j];
#pragma unroll
        for (int c = 0; c < K; ++c) acc[c] = fma(x, Bs[rr][c], acc[c]);
      }
    }
  }
  if (j < ncols) {
#pragma unroll
    for (int c = 0; c < K; ++c)
      if (c < k) P[((int64_t)blockIdx.y * k + c) * ncols + j] = acc[c];
  }
}

// C[j + c ldc] = sum over segments s = 0.. in order of P[s][c][j]
__global__ void k_rr_sum_segments(const double* P, int nseg, int ncols, int k, double* C, int ldc) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)ncols * k) return;
  const int c = (int)(e / ncols), j = (int)(e - (int64_t)c * ncols);
  double s = P[(int64_t)c * ncols + j];
  for (int g = 1; g < nseg; ++g) s += P[((int64_t)g * k + c) * ncols + j];
  C[(int64_t)c * ldc + j] = s;
}

// C (nws x k) = X B, B ncols x k: a warp per row of X, lanes over its columns,
// lane sums reduced by a shuffle tree (lane 0's result is written)
template <int K>
__global__ void __launch_bounds__(256) k_rr_xb(const double* X, int nws, int ncols, const double* B, int ldb,
                                               int k, double* C, int ldc) {
  const int row = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (row >= nws) return;  // whole warps
  double acc[K];
#pragma unroll
  for (int c = 0; c < K; ++c) acc[c] = 0.0;
  const double* x = X + (int64_t)row * ncols;
  for (int j = lane; j < ncols; j += 32) {
    const double xv = x[j];
#pragma unroll
    for (int c = 0; c < K; ++c)
      if (c < k) acc[c] = fma(xv, B[(int64_t)c * ldb + j], acc[c]);
  }
#pragma unroll
  for (int c = 0; c < K; ++c) {
    if (c < k) {
      double v = acc[c];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (lane == 0) C[(int64_t)c * ldc + row] = v;
    }
  }
}

// C (rows x k) = A (rows x k) W (k x k, ld k): a thread per entry, sum in order
__global__ void k_rr_small(const double* A, int lda, int rows, int k, const double* W, double* C, int ldc) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)rows * k) return;
  const int c = (int)(e / rows), i = (int)(e - (int64_t)c * rows);
  double s = 0.0;
  for (int l = 0; l < k; ++l) s = fma(A[(int64_t)l * lda + i], W[l + c * k], s);
  C[(int64_t)c * ldc + i] = s;
}

// block-wide sum of v (fixed order: a shuffle tree per warp, then the warps in
// order by thread 0); every thread returns it.  red: 33 doubles of shared memory
__device__ double rr_block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = red[0];
    for (int w = 1; w < nw; ++w) s += red[w];
    red[32] = s;
  }
  __syncthreads();
  return red[32];
}

// Orthonormal columns in place: A (rows x k, ld lda) = Q R by classical
// Gram-Schmidt applied twice per column (orthogonal to working precision); R
// (k x k, ld k, upper triangular, may be null) receives both passes'
// coefficients and the norms.  A column that the second pass shrinks below
// half its length lies in the span of the earlier ones to working precision
// (what is left is rounding, which no further pass makes orthogonal): it
// becomes zero, as does a zero column (R's diagonal 0).  One CTA.
template <int K>
__global__ void __launch_bounds__(256) k_rr_cgs2(double* A, int rows, int k, int lda, double* R) {
  __shared__ double red[33];
  __shared__ double wsum[8][K];
  __shared__ double d[K];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  if (R)
    for (int e = tid; e < k * k; e += blockDim.x) R[e] = 0.0;
  __syncthreads();
  for (int j = 0; j < k; ++j) {
    double* aj = A + (int64_t)j * lda;
    double n1 = 0.0;  // length after the first pass
    for (int pass = 0; pass < 2 && j > 0; ++pass) {
      double part[K];
#pragma unroll
      for (int i = 0; i < K; ++i) part[i] = 0.0;
      for (int row = tid; row < rows; row += blockDim.x) {
        const double v = aj[row];
#pragma unroll
        for (int i = 0; i < K; ++i)
          if (i < j) part[i] = fma(A[(int64_t)i * lda + row], v, part[i]);
      }
#pragma unroll
      for (int i = 0; i < K; ++i) {
        if (i < j) {
          double v = part[i];
          for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
          if (lane == 0) wsum[warp][i] = v;
        }
      }
      __syncthreads();
      if (tid < j) {
        double s = wsum[0][tid];
        for (int w = 1; w < nw; ++w) s += wsum[w][tid];
        d[tid] = s;
        if (R) R[tid + j * k] += s;
      }
      __syncthreads();
      for (int row = tid; row < rows; row += blockDim.x) {
        double v = aj[row];
        for (int i = 0; i < j; ++i) v = fma(-d[i], A[(int64_t)i * lda + row], v);
        aj[row] = v;
      }
      __syncthreads();
      if (pass == 0) {
        double t2 = 0.0;
        for (int row = tid; row < rows; row += blockDim.x) t2 = fma(aj[row], aj[row], t2);
        n1 = sqrt(rr_block_sum(t2, red));
      }
    }
    double s2 = 0.0;
    for (int row = tid; row < rows; row += blockDim.x) s2 = fma(aj[row], aj[row], s2);
    const double n2 = sqrt(rr_block_sum(s2, red));
    const double nrm = (j > 0 && n2 < 0.5 * n1) ? 0.0 : n2;
    if (R && tid == 0) R[j + j * k] = nrm;
    for (int row = tid; row < rows; row += blockDim.x) aj[row] = nrm > 0.0 ? aj[row] / nrm : 0.0;
    __syncthreads();
  }
}

// One-sided Jacobi SVD of the k x k matrix W (ld k, destroyed): its columns are
// rotated until pairwise orthogonal (|w_p . w_q| <= k eps |w_p| |w_q|), the
// rotations accumulated in V; then W_in = U diag(S) V^T.  Outputs sorted by
// descending singular value (ties: lower column first): S (k), U and Vs (k x k,
// ld k; a zero singular value gives a zero U column).  Rounds of disjoint
// pairs (a round-robin tournament over the columns), a warp per pair, each
// warp's reductions broadcast from lane 0 so all lanes rotate alike.  One CTA.
__global__ void __launch_bounds__(256) k_rr_jacobi(double* W, double* V, int k, double* S, double* U, double* Vs,
                                                   int* sweeps) {
  __shared__ int rotated;
  __shared__ double sv[kRrMaxK];
  __shared__ int order[kRrMaxK];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  for (int e = tid; e < k * k; e += blockDim.x) V[e] = (e % k == e / k) ? 1.0 : 0.0;
  const int kk = k + (k & 1);  // players (index k: a bye)
  const double tol = (double)k * 2.220446049250313e-16;
  int sweep = 0;
  for (; sweep < kRrMaxSweeps; ++sweep) {
    if (tid == 0) rotated = 0;
    __syncthreads();
    for (int round = 0; round < kk - 1; ++round) {
      for (int pi = warp; pi < kk / 2; pi += nw) {
        // position 0 holds player 0, position i >= 1 player 1 + (i - 1 + round) mod (kk - 1)
        const int ia = pi, ib = kk - 1 - pi;
        const int pa = ia == 0 ? 0 : 1 + (ia - 1 + round) % (kk - 1);
        const int pb = 1 + (ib - 1 + round) % (kk - 1);
        if (pa >= k || pb >= k) continue;
        const int p = min(pa, pb), q = max(pa, pb);
        double* wp = W + p * k;
        double* wq = W + q * k;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int r = lane; r < k; r += 32) {
          al = fma(wp[r], wp[r], al);
          be = fma(wq[r], wq[r], be);
          ga = fma(wp[r], wq[r], ga);
        }
        for (int o = 16; o > 0; o >>= 1) {
          al += __shfl_xor_sync(0xffffffffu, al, o);
          be += __shfl_xor_sync(0xffffffffu, be, o);
          ga += __shfl_xor_sync(0xffffffffu, ga, o);
        }
        al = __shfl_sync(0xffffffffu, al, 0);
        be = __shfl_sync(0xffffffffu, be, 0);
        ga = __shfl_sync(0xffffffffu, ga, 0);
        if (!(fabs(ga) > tol * sqrt(al) * sqrt(be))) continue;
        const double zeta = (be - al) / (2.0 * ga);
        const double t = fabs(zeta) > 1e150 ? 0.5 / zeta
                                            : copysign(1.0, zeta) / (fabs(zeta) + sqrt(fma(zeta, zeta, 1.0)));
        const double c = 1.0 / sqrt(fma(t, t, 1.0)), s = c * t;
        double* vp = V + p * k;
        double* vq = V + q * k;
        for (int r = lane; r < k; r += 32) {
          const double a = wp[r], b = wq[r];
          wp[r] = c * a - s * b;
          wq[r] = s * a + c * b;
          const double va = vp[r], vb = vq[r];
          vp[r] = c * va - s * vb;
          vq[r] = s * va + c * vb;
        }
        if (lane == 0) rotated = 1;
      }
      __syncthreads();
    }
    const int any = rotated;
    __syncthreads();
    if (!any) break;
  }
  for (int j = tid; j < k; j += blockDim.x) {
    double s2 = 0.0;
    for (int r = 0; r < k; ++r) s2 = fma(W[j * k + r], W[j * k + r], s2);
    sv[j] = sqrt(s2);
  }
  __syncthreads();
  if (tid == 0) {
    for (int j = 0; j < k; ++j) order[j] = j;
    for (int a = 0; a < k; ++a) {
      int best = a;
      for (int b = a + 1; b < k; ++b)
        if (sv[order[b]] > sv[order[best]] || (sv[order[b]] == sv[order[best]] && order[b] < order[best])) best = b;
      const int tmp = order[a];
      order[a] = order[best];
      order[best] = tmp;
    }
    if (sweeps) *sweeps = sweep;
  }
  __syncthreads();
  for (int e = tid; e < k * k; e += blockDim.x) {
    const int c = e / k, r = e - c * k, src = order[c];
    const double s = sv[src];
    if (r == 0) S[c] = s;
    U[e] = s > 0.0 ? W[src * k + r] / s : 0.0;
    Vs[e] = V[src * k + r];
  }
}

// partial sums of squares of the residual X - Q Bt^T (Q nws x k, Bt ncols x
// k): a thread per column j over a row segment, one partial per CTA
template <int K>
__global__ void __launch_bounds__(128) k_rr_resid(const double* X, int nws, int ncols, const double* Q,
                                                  const double* Bt, int k, int seg_rows, double* part) {
  __shared__ double Qs[32][K];
  __shared__ double red[33];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i0 = blockIdx.y * seg_rows, i1 = min(nws, i0 + seg_rows);
  double b[K];
#pragma unroll
  for (int c = 0; c < K; ++c) b[c] = (j < ncols && c < k) ? Bt[(int64_t)c * ncols + j] : 0.0;
  double ssq = 0.0;
  for (int it = i0; it < i1; it += 32) {
    const int nrow = min(32, i1 - it);
    __syncthreads();
    for (int e = threadIdx.x; e < 32 * K; e += blockDim.x) {
      const int rr = e / K, c = e - rr * K;
      Qs[rr][c] = (rr < nrow && c < k) ? Q[(int64_t)c * nws + it + rr] : 0.0;
    }
    __syncthreads();
    if (j < ncols) {
      for (int rr = 0; rr < nrow; ++rr) {
        double v = X[(int64_t)(it + rr) * ncols + j];
#pragma unroll
        for (int c = 0; c < K; ++c) v = fma(-Qs[rr][c], b[c], v);
        ssq = fma(v, v, ssq);
      }
    }
  }
  const double s = rr_block_sum(ssq, red);
  if (threadIdx.x == 0) part[(int64_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
}

// out[slot] = sum of v[0..n) in order (one thread: a few hundred partials)
__global__ void k_rr_sum_serial(const double* v, int n, double* out, int slot) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += v[i];
  out[slot] = s;
}

// out[slot] = sum of squares of v[0..n), one CTA, fixed order
__global__ void __launch_bounds__(256) k_rr_sumsq(const double* v, int n, double* out, int slot) {
  __shared__ double red[33];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s = fma(v[i], v[i], s);
  s = rr_block_sum(s, red);
  if (threadIdx.x == 0) out[slot] = s;
}

struct SvdWork {
  int kmax = 0;      // columns the buffers hold
  int ncols_max = 0;
  double *Om = nullptr, *Q = nullptr, *Z = nullptr, *Bt = nullptr, *L = nullptr, *Ub = nullptr;
  double *R = nullptr, *V = nullptr, *U = nullptr, *Vs = nullptr, *S = nullptr;
  double* P = nullptr;     // segment partials: kRrSegs x ncols_max x kmax
  double* part = nullptr;  // residual partials
  int part_cap = 0;
  double* scal = nullptr;  // device: [0] residual^2, [1] |mean|^2
  double hscal[3] = {0.0, 0.0, 0.0};  // host copy of scal and S[0]
  int* sweeps = nullptr;
};

constexpr int kRrSegs = 16;  // row segments of the X^T B products at most

int rr_bucket(int k) { return k <= 16 ? 16 : (k <= 32 ? 32 : 64); }

// row segments for X^T B / the residual: enough CTAs to cover the SMs
void rr_segments(int nws, int ncols, int* nseg, int* seg_rows) {
  const int colblocks = (ncols + 127) / 128;
  int s = std::max(1, std::min(kRrSegs, (296 + colblocks - 1) / colblocks));
  s = std::min(s, (nws + 31) / 32);
  int rows = (nws + s - 1) / s;
  rows = (rows + 31) / 32 * 32;
  *seg_rows = rows;
  *nseg = (nws + rows - 1) / rows;
}

// C (ncols x k, ld ncols) = X^T B (B nws x k, ld nws)
e2e_status rr_xtb(SvdWork& w, const double* X, int nws, int ncols, const double* B, int k, double* C,
                  cudaStream_t st) {
  int nseg, seg_rows;
  rr_segments(nws, ncols, &nseg, &seg_rows);
  const dim3 grid((unsigned)((ncols + 127) / 128), (unsigned)nseg);
  switch (rr_bucket(k)) {
    case 16: k_rr_xtb<16><<<grid, 128, 0, st>>>(X, nws, ncols, B, nws, k, seg_rows, w.P); break;
    case 32: k_rr_xtb<32><<<grid, 128, 0, st>>>(X, nws, ncols, B, nws, k, seg_rows, w.P); break;
    default: k_rr_xtb<64><<<grid, 128, 0, st>>>(X, nws, ncols, B, nws, k, seg_rows, w.P); break;
  }
  CK(cudaGetLastError());
  const int64_t ne = (int64_t)ncols * k;
  k_rr_sum_segments<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(w.P, nseg, ncols, k, C, ncols);
  CK(cudaGetLastError());
  return E2E_OK;
}

// C (nws x k, ld nws) = X B (B ncols x k, ld ncols)
e2e_status rr_xb(const double* X, int nws, int ncols, const double* B, int k, double* C, cudaStream_t st) {
  const unsigned blocks = (unsigned)(((int64_t)nws * 32 + 255) / 256);
  switch (rr_bucket(k)) {
    case 16: k_rr_xb<16><<<blocks, 256, 0, st>>>(X, nws, ncols, B, ncols, k, C, nws); break;
    case 32: k_rr_xb<32><<<blocks, 256, 0, st>>>(X, nws, ncols, B, ncols, k, C, nws); break;
    default: k_rr_xb<64><<<blocks, 256, 0, st>>>(X, nws, ncols, B, ncols, k, C, nws); break;
  }
  CK(cudaGetLastError());
  return E2E_OK;
}

e2e_status rr_orth(double* A, int rows, int k, double* R, cudaStream_t st) {
  switch (rr_bucket(k)) {
    case 16: k_rr_cgs2<16><<<1, 256, 0, st>>>(A, rows, k, rows, R); break;
    case 32: k_rr_cgs2<32><<<1, 256, 0, st>>>(A, rows, k, rows, R); break;
    default: k_rr_cgs2<64><<<1, 256, 0, st>>>(A, rows, k, rows, R); break;
  }
  CK(cudaGetLastError());
  return E2E_OK;
}

// |X - Q Bt^T|_F^2 into w.scal[0]
e2e_status rr_residual(SvdWork& w, const double* X, int nws, int ncols, int k, cudaStream_t st) {
  int nseg, seg_rows;
  rr_segments(nws, ncols, &nseg, &seg_rows);
  const dim3 grid((unsigned)((ncols + 127) / 128), (unsigned)nseg);
  const int np = (int)(grid.x * grid.y);
  if (np > w.part_cap) return fail(E2E_ERR_INVALID, "residual partials above capacity");
  switch (rr_bucket(k)) {
    case 16: k_rr_resid<16><<<grid, 128, 0, st>>>(X, nws, ncols, w.Q, w.Bt, k, seg_rows, w.part); break;
    case 32: k_rr_resid<32><<<grid, 128, 0, st>>>(X, nws, ncols, w.Q, w.Bt, k, seg_rows, w.part); break;
    default: k_rr_resid<64><<<grid, 128, 0, st>>>(X, nws, ncols, w.Q, w.Bt, k, seg_rows, w.part); break;
  }
  CK(cudaGetLastError());
  k_rr_sum_serial<<<1, 32, 0, st>>>(w.part, np, w.scal, 0);
  CK(cudaGetLastError());
  return E2E_OK;
}

// Randomized SVD of the centred X (row-major nws x ncols) with k columns and
// `power` power iterations; *ok when certified:
//  * |X - Q Q^T X|_F <= 1e-10 s_1 (then each kept singular value is exact to
//    about |R|^2 / s_k, machine precision relative to s_1), or
//  * s_1 <= 1e-10 sqrt(nws) |mean|: the centred matrix is below the rounding of
//    the data it was centred from (every realisation alike, as at t = 0), so
//    its singular vectors are not determined by the data and the computed ones
//    stand, as LAPACK's do for the reference.
e2e_status randomized_svd(SvdWork& w, const double* X, int nws, int ncols, int r, int k, int power,
                          const double* mean, double* C, double* M, double* svals, bool* ok, cudaStream_t st) {
  *ok = false;
  const int64_t no = (int64_t)ncols * k;
  k_env_test_matrix<<<(unsigned)((no + 255) / 256), 256, 0, st>>>(w.Om, no);
  CK(cudaGetLastError());
  e2e_status s;
  if ((s = rr_xb(X, nws, ncols, w.Om, k, w.Q, st)) != E2E_OK) return s;     // Q = X Om
  if ((s = rr_orth(w.Q, nws, k, nullptr, st)) != E2E_OK) return s;
  for (int it = 0; it < power; ++it) {                                        // Q <- orth(X orth(X^T Q))
    if ((s = rr_xtb(w, X, nws, ncols, w.Q, k, w.Z, st)) != E2E_OK) return s;
    if ((s = rr_orth(w.Z, ncols, k, nullptr, st)) != E2E_OK) return s;
    if ((s = rr_xb(X, nws, ncols, w.Z, k, w.Q, st)) != E2E_OK) return s;
    if ((s = rr_orth(w.Q, nws, k, nullptr, st)) != E2E_OK) return s;
  }
  if ((s = rr_xtb(w, X, nws, ncols, w.Q, k, w.Bt, st)) != E2E_OK) return s;  // Bt = X^T Q
  if ((s = rr_residual(w, X, nws, ncols, k, st)) != E2E_OK) return s;
  k_rr_sumsq<<<1, 256, 0, st>>>(mean, ncols, w.scal, 1);
  CK(cudaGetLastError());
  // Bt = Qb R (Bt becomes Qb), R = U_R S V_R^T, Ub = Qb U_R, L = Q V_R
  if ((s = rr_orth(w.Bt, ncols, k, w.R, st)) != E2E_OK) return s;
  k_rr_jacobi<<<1, 256, 0, st>>>(w.R, w.V, k, w.S, w.U, w.Vs, w.sweeps);
  CK(cudaGetLastError());
  const int64_t nu = (int64_t)ncols * k, nl = (int64_t)nws * k;
  k_rr_small<<<(unsigned)((nu + 255) / 256), 256, 0, st>>>(w.Bt, ncols, ncols, k, w.U, w.Ub, ncols);
  k_rr_small<<<(unsigned)((nl + 255) / 256), 256, 0, st>>>(w.Q, nws, nws, k, w.Vs, w.L, nws);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(w.hscal, w.scal, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(w.hscal + 2, w.S, sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const double rnorm = sqrt(w.hscal[0]), mnorm = sqrt(w.hscal[1]), s1 = w.hscal[2];
  const bool certified = (s1 > 0.0 && rnorm <= 1e-10 * s1) || !(s1 > 1e-10 * sqrt((double)nws) * mnorm);
  if (!certified || !std::isfinite(rnorm) || !std::isfinite(s1)) return E2E_OK;
  ModeArgs a;
  a.nws = nws;
  a.ncols = ncols;
  a.r = r;
  a.S = w.S;
  a.Us = w.L;
  a.ldu = nws;
  a.Vs = w.Ub;
  a.ldv = ncols;
  a.C = C;
  a.M = M;
  a.svals = svals;
  k_env_modes<<<r, 256, 0, st>>>(a);
  CK(cudaGetLastError());
  *ok = true;
  return E2E_OK;
}

// The leading r triplets: k = n_modes + 10 columns and two power iterations;
// if that is not certified, twice the columns (up to 64 and the matrix's
// smaller side) and four power iterations until it is.  When the columns span
// the whole smaller side the residual is rounding only, so only n_modes above
// 54 on a matrix wider than 64 can end uncertified: then an error.
e2e_status truncated_svd(SvdWork& w, const double* X, int nws, int ncols, int r, const double* mean, double* C,
                         double* M, double* svals, cudaStream_t st, int* enlarged) {
  const int nsmall = std::min(nws, ncols);
  int k = std::min(std::min(r + 10, kRrMaxK), nsmall), power = 2;
  if (k < r) return fail(E2E_ERR_UNSUPPORTED, "n_modes above the range finder's 64 columns");
  for (;;) {
    bool ok = false;
    e2e_status s = randomized_svd(w, X, nws, ncols, r, k, power, mean, C, M, svals, &ok, st);
    if (s != E2E_OK) return s;
    if (ok) return E2E_OK;
    const int k2 = std::min(std::min(2 * k, kRrMaxK), nsmall);
    if (k2 == k && power >= 4)
      return fail(E2E_ERR_DEVICE, "rank reduction not certified with " + std::to_string(k) +
                                      " columns (|X - QQ^T X| above 1e-10 s_1)");
    ++*enlarged;
    k = k2;
    power = 4;
  }
}

}  // namespace

extern "C" e2e_status e2e_env_generate(const e2e_env_params* p, const int32_t* interp_vertices,
                                       const double* interp_weights, int out_where, const e2e_env_fields* out,
                                       double* svals_out, e2e_env_stats* stats, void* stream) {
  if (!p || !out) return fail(E2E_ERR_INVALID, "null argument");
  if (out_where != E2E_HOST && out_where != E2E_DEVICE) return fail(E2E_ERR_INVALID, "bad out_where");
  const int g = p->init_gsize, nt = p->nt, nws = p->n_wsamples, r = p->n_modes, d = p->interpolate_degree;
  if (g < 2 || nt < 1 || nws < 2 || r < 1 || d < 1)
    return fail(E2E_ERR_INVALID, "init_gsize >= 2, nt >= 1, n_wsamples >= 2, n_modes >= 1, interpolate_degree >= 1");
  const int n = g * g;
  // the reference asserts n_modes <= min(nt, n_wsamples, 2 n) (:213); the scalar
  // field's reduction needs n_modes <= min(n_wsamples, n) as well
  if (r > nt || r > nws || r > n) return fail(E2E_ERR_INVALID, "n_modes above min(nt, n_wsamples, init_gsize^2)");
  if (!interp_vertices || !interp_weights) return fail(E2E_ERR_INVALID, "null interpolation table");
  if (p->obstacle_mode < E2E_OBST_NONE || p->obstacle_mode > E2E_OBST_DYNAMIC)
    return fail(E2E_ERR_INVALID, "bad obstacle_mode");
  if (!out->u || !out->v || !out->ui || !out->vi || !out->yi || !out->phi || !out->phi_i || !out->phi_yi ||
      !out->s || !out->mask)
    return fail(E2E_ERR_INVALID, "null output array");
  const int64_t G = (int64_t)g * d, G2 = G * G;
  if (G > 46340) return fail(E2E_ERR_UNSUPPORTED, "fine grid too large");
  if ((int64_t)nws * 2 * n > (int64_t)0x7fffffff)
    return fail(E2E_ERR_UNSUPPORTED, "n_wsamples x 2 init_gsize^2 above 2^31 (32-bit solver dimensions)");
  if (!(p->dxy > 0.0) || !(p->dt >= 0.0)) return fail(E2E_ERR_INVALID, "dxy must be positive and dt non-negative");
  cudaStream_t st = (cudaStream_t)stream;
  DeviceScratch scratch(st);

  cudaEvent_t ev[2];
  for (int k = 0; k < 2; ++k) CK(cudaEventCreate(&ev[k]));
  struct EvFree {
    cudaEvent_t* e;
    ~EvFree() { for (int k = 0; k < 2; ++k) cudaEventDestroy(e[k]); }
  } evfree{ev};
  CK(cudaEventRecord(ev[0], st));

  // the interpolation table on the device
  int32_t* dvert = nullptr;
  double* dwgt = nullptr;
  CK(dalloc((void**)&dvert, sizeof(int32_t) * 3 * (size_t)G2, st));
  scratch.add(dvert);
  CK(dalloc((void**)&dwgt, sizeof(double) * 3 * (size_t)G2, st));
  scratch.add(dwgt);
  CK(cudaMemcpyAsync(dvert, interp_vertices, sizeof(int32_t) * 3 * (size_t)G2, cudaMemcpyDefault, st));
  CK(cudaMemcpyAsync(dwgt, interp_weights, sizeof(double) * 3 * (size_t)G2, cudaMemcpyDefault, st));

  // per-step matrices and the results of all steps
  double *Xv, *Xp, *mv, *mp, *Cv, *Cp, *Mv, *Mp, *sv;
  double* coarse;
  float *yi, *phi_yi;
  const int nb = 3 + 3 * r;
  CK(dalloc((void**)&Xv, sizeof(double) * (size_t)nws * 2 * n, st));
  scratch.add(Xv);
  CK(dalloc((void**)&Xp, sizeof(double) * (size_t)nws * n, st));
  scratch.add(Xp);
  CK(dalloc((void**)&mv, sizeof(double) * 2 * (size_t)n, st));
  scratch.add(mv);
  CK(dalloc((void**)&mp, sizeof(double) * (size_t)n, st));
  scratch.add(mp);
  CK(dalloc((void**)&Cv, sizeof(double) * (size_t)nws * r, st));
  scratch.add(Cv);
  CK(dalloc((void**)&Cp, sizeof(double) * (size_t)nws * r, st));
  scratch.add(Cp);
  CK(dalloc((void**)&Mv, sizeof(double) * (size_t)r * 2 * n, st));
  scratch.add(Mv);
  CK(dalloc((void**)&Mp, sizeof(double) * (size_t)r * n, st));
  scratch.add(Mp);
  CK(dalloc((void**)&sv, sizeof(double) * 2 * (size_t)nt * r, st));
  scratch.add(sv);
  CK(dalloc((void**)&coarse, sizeof(double) * (size_t)nt * nb * n, st));
  scratch.add(coarse);

  // outputs (device: the caller's arrays; host: staged and copied at the end)
  e2e_env_fields o = *out;
  const size_t b2 = sizeof(float) * (size_t)nt * G2, bm = b2 * r, by = sizeof(float) * (size_t)nt * nws * r;
  if (out_where == E2E_HOST) {
    float** fp[9] = {&o.u, &o.v, &o.ui, &o.vi, &o.yi, &o.phi, &o.phi_i, &o.phi_yi, &o.s};
    const size_t fb[9] = {b2, b2, bm, bm, by, b2, bm, by, b2};
    for (int k = 0; k < 9; ++k) {
      CK(dalloc((void**)fp[k], fb[k], st));
      scratch.add(*fp[k]);
    }
    CK(dalloc((void**)&o.mask, sizeof(int32_t) * (size_t)nt * G2, st));
    scratch.add(o.mask);
  }
  yi = o.yi;
  phi_yi = o.phi_yi;

  // rank-reduction work space, sized for the wider (velocity) matrix and the
  // largest range finder
  SvdWork w;
  {
    w.kmax = kRrMaxK;
    w.ncols_max = 2 * n;
    const size_t kc = (size_t)w.ncols_max * w.kmax, ks = (size_t)nws * w.kmax, kk = (size_t)w.kmax * w.kmax;
    double** wide[] = {&w.Om, &w.Z, &w.Bt, &w.Ub};
    for (double** b : wide) {
      CK(dalloc((void**)b, sizeof(double) * kc, st));
      scratch.add(*b);
    }
    double** tall[] = {&w.Q, &w.L};
    for (double** b : tall) {
      CK(dalloc((void**)b, sizeof(double) * ks, st));
      scratch.add(*b);
    }
    double** sq[] = {&w.R, &w.V, &w.U, &w.Vs};
    for (double** b : sq) {
      CK(dalloc((void**)b, sizeof(double) * kk, st));
      scratch.add(*b);
    }
    CK(dalloc((void**)&w.S, sizeof(double) * w.kmax, st));
    scratch.add(w.S);
    CK(dalloc((void**)&w.P, sizeof(double) * kRrSegs * kc, st));
    scratch.add(w.P);
    w.part_cap = ((w.ncols_max + 127) / 128) * kRrSegs;
    CK(dalloc((void**)&w.part, sizeof(double) * w.part_cap, st));
    scratch.add(w.part);
    CK(dalloc((void**)&w.scal, sizeof(double) * 2, st));
    scratch.add(w.scal);
    CK(dalloc((void**)&w.sweeps, sizeof(int), st));
    scratch.add(w.sweeps);
  }
  int enlarged = 0;

  for (int t = 0; t < nt; ++t) {
    RealArgs ra{g, nws, t, (double)t * p->dt, p->dxy, p->A, p->eps, p->w_lo, p->w_hi, p->wx, 0.5 * kPi, Xv, Xp};
    const int64_t nr = (int64_t)nws * n;
    k_env_realisations<<<(unsigned)((nr + 255) / 256), 256, 0, st>>>(ra);
    CK(cudaGetLastError());
    k_env_center<<<(2 * n + 127) / 128, 128, 0, st>>>(Xv, nws, 2 * n, mv);
    k_env_center<<<(n + 127) / 128, 128, 0, st>>>(Xp, nws, n, mp);
    CK(cudaGetLastError());
    e2e_status s = truncated_svd(w, Xv, nws, 2 * n, r, mv, Cv, Mv, sv + (int64_t)t * r, st, &enlarged);
    if (s != E2E_OK) return s;
    s = truncated_svd(w, Xp, nws, n, r, mp, Cp, Mp, sv + (int64_t)(nt + t) * r, st, &enlarged);
    if (s != E2E_OK) return s;
    const int64_t ns = std::max<int64_t>((int64_t)nb * n, (int64_t)nws * r);
    k_env_store<<<(unsigned)((ns + 255) / 256), 256, 0, st>>>(n, nws, r, mv, mp, Mv, Mp, Cv, Cp,
                                                                coarse + (int64_t)t * nb * n,
                                                                yi + (int64_t)t * nws * r,
                                                                phi_yi + (int64_t)t * nws * r);
    CK(cudaGetLastError());
  }
  unsigned int* derr = nullptr;
  CK(dalloc((void**)&derr, sizeof(unsigned int), st));
  scratch.add(derr);
  CK(cudaMemsetAsync(derr, 0, sizeof(unsigned int), st));
  InterpArgs ia{nt, r, n, (int)G2, coarse, dvert, dwgt, derr, o.u, o.v, o.phi, o.ui, o.vi, o.phi_i};
  const int64_t ni = (int64_t)nt * nb * G2;
  k_env_interpolate<<<(unsigned)((ni + 255) / 256), 256, 0, st>>>(ia);
  CK(cudaGetLastError());
  CloudArgs ca{nt, (int)G, p->dxy / d, p->A_sc, p->obstacle_mode, p->obs_upper_row, p->obs_left_col,
               p->obs_width, p->obs_speed_x, p->obs_speed_y, o.s, o.mask};
  const int64_t nc = (int64_t)nt * G2;
  k_env_cloud<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(ca);
  CK(cudaGetLastError());
  CK(cudaEventRecord(ev[1], st));

  if (out_where == E2E_HOST) {
    float* const* fp[9] = {&o.u, &o.v, &o.ui, &o.vi, &o.yi, &o.phi, &o.phi_i, &o.phi_yi, &o.s};
    float* const hp[9] = {out->u, out->v, out->ui, out->vi, out->yi, out->phi, out->phi_i, out->phi_yi, out->s};
    const size_t fb[9] = {b2, b2, bm, bm, by, b2, bm, by, b2};
    for (int k = 0; k < 9; ++k) CK(cudaMemcpyAsync(hp[k], *fp[k], fb[k], cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(out->mask, o.mask, sizeof(int32_t) * (size_t)nt * G2, cudaMemcpyDeviceToHost, st));
  }
  if (svals_out) CK(cudaMemcpyAsync(svals_out, sv, sizeof(double) * 2 * (size_t)nt * r, cudaMemcpyDefault, st));
  unsigned int herr = 0;
  CK(cudaMemcpyAsync(&herr, derr, sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (herr) return fail(E2E_ERR_INVALID, "interpolation table: a vertex index outside the coarse grid");
  if (stats) {
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    stats->seconds = ms * 1e-3;
    stats->fine_gsize = (int32_t)G;
    stats->transposed_vel = 0;
    stats->transposed_phi = 0;
    stats->full_svds = enlarged;
  }
  return E2E_OK;
}
