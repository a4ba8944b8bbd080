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
//   SVD                 of the centred matrix, the leading n_modes triplets:
//                       a randomized range finder (n_modes + 10 columns, two
//                       power iterations, QR by cuSOLVER, products by cuBLAS)
//                       and a one-sided Jacobi SVD (cuSOLVER gesvdj) of the
//                       projected matrix, accepted when the explicit residual
//                       |X - Q Q^T X|_F is below 1e-10 s_1 (then every kept
//                       singular value is exact to ~|R|^2/s_k); otherwise, as
//                       at t = 0 where X is rounding noise, gesvdj of the whole
//                       matrix.  Either way singular values come to about
//                       machine precision relative to the largest, like
//                       np.linalg.svd's LAPACK (a Gram-matrix eigensolve would
//                       lose (s_1/s_k)^2 of it, and s_4/s_1 ~ 1e-6 here); the
//                       first n_modes give coefficients u_k s_k and modes v_k,
//                       signs fixed so that each coefficient column's
//                       largest-magnitude entry is positive (the reference's
//                       np.linalg.svd leaves the sign to LAPACK)
// then, for all steps, k_env_interpolate: the reference's griddata 'linear' on
// the coarse cell centres, evaluated from a table of (triangle vertices,
// barycentric weights) per fine point that the caller builds from the same
// Delaunay triangulation (scipy's), summed in griddata's order in double
// without contraction; points outside the hull read 0 (np.nan_to_num of the
// fill value).
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>
#include <math.h>

#include <algorithm>
#include <mutex>
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
#define CKB(call)                                                                               \
  do {                                                                                          \
    cublasStatus_t _s = (call);                                                                 \
    if (_s != CUBLAS_STATUS_SUCCESS)                                                            \
      return fail(E2E_ERR_CUDA, std::string(#call) + ": cuBLAS status " + std::to_string((int)_s)); \
  } while (0)
#define CKS(call)                                                                           \
  do {                                                                                      \
    cusolverStatus_t _s = (call);                                                           \
    if (_s != CUSOLVER_STATUS_SUCCESS)                                                      \
      return fail(E2E_ERR_CUDA, std::string(#call) + ": cuSOLVER status " + std::to_string((int)_s)); \
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

// row-major nws x ncols -> column-major (ld nws)
__global__ void k_env_transpose(const double* X, int nws, int ncols, double* B) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)nws * ncols) return;
  const int k = (int)(idx / ncols), c = (int)(idx - (int64_t)k * ncols);
  B[(int64_t)c * nws + k] = X[idx];
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

// Truncated SVD of the centred nws x ncols matrix X (row-major, on the device;
// destroyed) by one-sided Jacobi (cuSOLVER gesvdj, economy size, sorted): the
// row-major buffer is the column-major ncols x nws matrix X^T, which gesvdj
// takes directly when ncols >= nws (X^T = U S V^T: X's left vectors are V);
// otherwise X is transposed into column-major nws x ncols first.
// cuSOLVER and cuBLAS handles, one pair per device for the whole process,
// created on first use and kept until exit (never destroyed: a destructor at
// process exit could run after the CUDA context is gone).  A call holds the
// device's mutex while it uses them, so calls from any number of host
// threads share one pair and one work space; generations on one device run
// one at a time.  Creating the handles on every call allocated their device
// work space through the driver each time, which on a busy machine added tens
// of milliseconds to a 35 ms generation.  The handles belong to the device's
// primary context: after cudaDeviceReset the process must not generate again.
struct DevHandles {
  std::mutex mu;
  cusolverDnHandle_t sol = nullptr;
  cublasHandle_t blas = nullptr;
};
DevHandles g_handles[64];

e2e_status solver_handles(cusolverDnHandle_t* sol, cublasHandle_t* blas, std::unique_lock<std::mutex>* hold) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return fail(E2E_ERR_UNSUPPORTED, "device index above 63");
  DevHandles& x = g_handles[dev];
  std::unique_lock<std::mutex> lk(x.mu);
  if (!x.sol && cusolverDnCreate(&x.sol) != CUSOLVER_STATUS_SUCCESS) {
    x.sol = nullptr;
    return fail(E2E_ERR_CUDA, "cusolverDnCreate");
  }
  if (!x.blas && cublasCreate(&x.blas) != CUBLAS_STATUS_SUCCESS) {
    x.blas = nullptr;
    return fail(E2E_ERR_CUDA, "cublasCreate");
  }
  *sol = x.sol;
  *blas = x.blas;
  *hold = std::move(lk);
  return E2E_OK;
}

struct SvdWork {
  cusolverDnHandle_t sol = nullptr;
  cublasHandle_t blas = nullptr;
  gesvdjInfo_t params = nullptr;
  // randomized range finder: k = r + oversampling columns
  int k = 0;
  double *Om = nullptr, *Q = nullptr, *Z = nullptr, *Bt = nullptr, *L = nullptr, *R = nullptr;
  double *Ub = nullptr, *Vb = nullptr, *Sb = nullptr, *tau = nullptr;
  double* qwork = nullptr;
  int lqwork = 0;
  double* B = nullptr;  // transposed copy (nws > ncols)
  double* U = nullptr;  // m x min(m, n)
  double* V = nullptr;  // n x min(m, n)
  double* S = nullptr;  // min(m, n)
  double* work = nullptr;
  int lwork = 0;
  int* info = nullptr;
};

e2e_status svd_shape(int nws, int ncols, int* m, int* n) {
  if (ncols >= nws) {
    *m = ncols;
    *n = nws;
  } else {
    *m = nws;
    *n = ncols;
  }
  return E2E_OK;
}

// orthonormal basis of the column range of A (rows x k, column-major, ld rows), in place
e2e_status orthonormalize(SvdWork& w, double* A, int rows, int k) {
  CKS(cusolverDnDgeqrf(w.sol, rows, k, A, rows, w.tau, w.qwork, w.lqwork, w.info));
  CKS(cusolverDnDorgqr(w.sol, rows, k, k, A, rows, w.tau, w.qwork, w.lqwork, w.info));
  return E2E_OK;
}

// Randomized SVD of X (row-major nws x ncols, read only).  Returns false in
// *ok when the residual check fails (the caller then runs gesvdj).
e2e_status randomized_svd(SvdWork& w, const double* X, int nws, int ncols, int r, double* C, double* M,
                          double* svals, bool* ok, cudaStream_t st) {
  *ok = false;
  const int k = std::min(w.k, std::min(nws, ncols));
  if (k <= r || (int64_t)nws * ncols > (int64_t)0x7fffffff) return E2E_OK;
  const double one = 1.0, zero = 0.0, mone = -1.0;
  // X as the column-major ncols x nws matrix Xc (= X^T), ld ncols
  const int64_t no = (int64_t)ncols * k;
  k_env_test_matrix<<<(unsigned)((no + 255) / 256), 256, 0, st>>>(w.Om, no);
  CK(cudaGetLastError());
  // Q = X Om (nws x k)
  CKB(cublasDgemm(w.blas, CUBLAS_OP_T, CUBLAS_OP_N, nws, k, ncols, &one, X, ncols, w.Om, ncols, &zero, w.Q, nws));
  e2e_status s = orthonormalize(w, w.Q, nws, k);
  if (s != E2E_OK) return s;
  for (int it = 0; it < 2; ++it) {  // power iterations: Q <- orth(X orth(X^T Q))
    CKB(cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, ncols, k, nws, &one, X, ncols, w.Q, nws, &zero, w.Z, ncols));
    s = orthonormalize(w, w.Z, ncols, k);
    if (s != E2E_OK) return s;
    CKB(cublasDgemm(w.blas, CUBLAS_OP_T, CUBLAS_OP_N, nws, k, ncols, &one, X, ncols, w.Z, ncols, &zero, w.Q, nws));
    s = orthonormalize(w, w.Q, nws, k);
    if (s != E2E_OK) return s;
  }
  // Bt = X^T Q (ncols x k) = (Q^T X)^T
  CKB(cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, ncols, k, nws, &one, X, ncols, w.Q, nws, &zero, w.Bt, ncols));
  // residual X - Q Q^T X, as Xc - Bt Q^T, and its Frobenius norm
  CK(cudaMemcpyAsync(w.R, X, sizeof(double) * (size_t)nws * ncols, cudaMemcpyDeviceToDevice, st));
  CKB(cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_T, ncols, nws, k, &mone, w.Bt, ncols, w.Q, nws, &one, w.R, ncols));
  double rnorm = 0.0;
  CKB(cublasDnrm2(w.blas, nws * ncols, w.R, 1, &rnorm));  // host result: synchronises
  // SVD of the tall Bt = Ub S Vb^T: X ~ Q B = (Q Vb) S Ub^T
  CKS(cusolverDnDgesvdj(w.sol, CUSOLVER_EIG_MODE_VECTOR, 1, ncols, k, w.Bt, ncols, w.Sb, w.Ub, ncols, w.Vb, k,
                        w.work, w.lwork, w.info, w.params));
  int h_info = 0;
  CK(cudaMemcpyAsync(&h_info, w.info, sizeof(int), cudaMemcpyDeviceToHost, st));
  double s1 = 0.0;
  CK(cudaMemcpyAsync(&s1, w.Sb, sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (h_info != 0 || !(rnorm <= 1e-10 * s1) || !(s1 > 0.0)) return E2E_OK;
  CKB(cublasDgemm(w.blas, CUBLAS_OP_N, CUBLAS_OP_N, nws, k, k, &one, w.Q, nws, w.Vb, k, &zero, w.L, nws));
  ModeArgs a;
  a.nws = nws;
  a.ncols = ncols;
  a.r = r;
  a.S = w.Sb;
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

e2e_status truncated_svd(SvdWork& w, double* X, int nws, int ncols, int r, double* C, double* M, double* svals,
                         cudaStream_t st, int* full_svds) {
  bool ok = false;
  e2e_status rs = randomized_svd(w, X, nws, ncols, r, C, M, svals, &ok, st);
  if (rs != E2E_OK) return rs;
  if (ok) return E2E_OK;
  ++*full_svds;
  int m, n;
  svd_shape(nws, ncols, &m, &n);
  double* A = X;
  if (ncols < nws) {
    const int64_t tot = (int64_t)nws * ncols;
    k_env_transpose<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(X, nws, ncols, w.B);
    CK(cudaGetLastError());
    A = w.B;
  }
  CKS(cusolverDnDgesvdj(w.sol, CUSOLVER_EIG_MODE_VECTOR, 1, m, n, A, m, w.S, w.U, m, w.V, n, w.work, w.lwork, w.info,
                        w.params));
  int h_info = 0;
  CK(cudaMemcpyAsync(&h_info, w.info, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (h_info != 0) return fail(E2E_ERR_DEVICE, "Jacobi SVD did not converge (info " + std::to_string(h_info) + ")");
  ModeArgs a;
  a.nws = nws;
  a.ncols = ncols;
  a.r = r;
  a.S = w.S;
  if (ncols >= nws) {  // X^T = U S V^T: sample side V (n = nws rows), grid side U (m = ncols rows)
    a.Us = w.V;
    a.ldu = n;
    a.Vs = w.U;
    a.ldv = m;
  } else {             // X = U S V^T: sample side U (m = nws rows), grid side V (n = ncols rows)
    a.Us = w.U;
    a.ldu = m;
    a.Vs = w.V;
    a.ldv = n;
  }
  a.C = C;
  a.M = M;
  a.svals = svals;
  k_env_modes<<<r, 256, 0, st>>>(a);
  CK(cudaGetLastError());
  return E2E_OK;
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

  // Jacobi SVD work space (the larger of the two reductions)
  SvdWork w;
  struct SvdFree {
    SvdWork* w;
    ~SvdFree() {
      if (w->params) cusolverDnDestroyGesvdjInfo(w->params);
    }
  } svdfree{&w};
  std::unique_lock<std::mutex> handles_held;  // the device's handles, until this call returns
  {
    e2e_status hs = solver_handles(&w.sol, &w.blas, &handles_held);
    if (hs != E2E_OK) return hs;
  }
  // on every return, the work queued with the handles finishes before the
  // next caller may set them to its own stream
  struct DrainBeforeRelease {
    cudaStream_t s;
    ~DrainBeforeRelease() { cudaStreamSynchronize(s); }
  } drain{st};
  CKS(cusolverDnSetStream(w.sol, st));
  CKB(cublasSetStream(w.blas, st));
  CKB(cublasSetPointerMode(w.blas, CUBLAS_POINTER_MODE_HOST));
  CKS(cusolverDnCreateGesvdjInfo(&w.params));
  CKS(cusolverDnXgesvdjSetSortEig(w.params, 1));
  {
    size_t bu = 0, bv = 0, bs = 0, bb = 0;
    for (int ncols : {2 * n, n}) {
      int m, k;
      svd_shape(nws, ncols, &m, &k);
      bu = std::max(bu, (size_t)m * k);
      bv = std::max(bv, (size_t)k * k);
      bs = std::max(bs, (size_t)k);
      if (ncols < nws) bb = std::max(bb, (size_t)nws * ncols);
    }
    CK(dalloc((void**)&w.U, sizeof(double) * bu, st));
    scratch.add(w.U);
    CK(dalloc((void**)&w.V, sizeof(double) * bv, st));
    scratch.add(w.V);
    CK(dalloc((void**)&w.S, sizeof(double) * bs, st));
    scratch.add(w.S);
    if (bb) {
      CK(dalloc((void**)&w.B, sizeof(double) * bb, st));
      scratch.add(w.B);
    }
    CK(dalloc((void**)&w.info, sizeof(int), st));
    scratch.add(w.info);
    for (int ncols : {2 * n, n}) {
      int m, k, lw = 0;
      svd_shape(nws, ncols, &m, &k);
      CKS(cusolverDnDgesvdj_bufferSize(w.sol, CUSOLVER_EIG_MODE_VECTOR, 1, m, k, Xv, m, w.S, w.U, m, w.V, k, &lw,
                                       w.params));
      w.lwork = std::max(w.lwork, lw);
    }
    // randomized range finder: k = n_modes + 10 columns
    w.k = std::min(r + 10, std::min(nws, n));
    const int kk = w.k, cmax = std::max(2 * n, nws);
    double** rb[] = {&w.Om, &w.Z, &w.Bt, &w.Ub, &w.Q, &w.L};
    for (double** b : rb) {
      CK(dalloc((void**)b, sizeof(double) * (size_t)cmax * kk, st));
      scratch.add(*b);
    }
    CK(dalloc((void**)&w.R, sizeof(double) * (size_t)nws * 2 * n, st));
    scratch.add(w.R);
    CK(dalloc((void**)&w.Vb, sizeof(double) * (size_t)kk * kk, st));
    scratch.add(w.Vb);
    CK(dalloc((void**)&w.Sb, sizeof(double) * (size_t)kk, st));
    scratch.add(w.Sb);
    CK(dalloc((void**)&w.tau, sizeof(double) * (size_t)kk, st));
    scratch.add(w.tau);
    for (int rows : {nws, 2 * n, n}) {
      int lw = 0;
      CKS(cusolverDnDgeqrf_bufferSize(w.sol, rows, kk, w.Q, rows, &lw));
      w.lqwork = std::max(w.lqwork, lw);
      CKS(cusolverDnDorgqr_bufferSize(w.sol, rows, kk, kk, w.Q, rows, w.tau, &lw));
      w.lqwork = std::max(w.lqwork, lw);
    }
    for (int ncols : {2 * n, n}) {
      int lw = 0;
      CKS(cusolverDnDgesvdj_bufferSize(w.sol, CUSOLVER_EIG_MODE_VECTOR, 1, ncols, kk, w.Bt, ncols, w.Sb, w.Ub,
                                       ncols, w.Vb, kk, &lw, w.params));
      w.lwork = std::max(w.lwork, lw);
    }
    CK(dalloc((void**)&w.qwork, sizeof(double) * (size_t)std::max(w.lqwork, 1), st));
    scratch.add(w.qwork);
    CK(dalloc((void**)&w.work, sizeof(double) * (size_t)std::max(w.lwork, 1), st));
    scratch.add(w.work);
  }
  int full_svds = 0;

  for (int t = 0; t < nt; ++t) {
    RealArgs ra{g, nws, t, (double)t * p->dt, p->dxy, p->A, p->eps, p->w_lo, p->w_hi, p->wx, 0.5 * kPi, Xv, Xp};
    const int64_t nr = (int64_t)nws * n;
    k_env_realisations<<<(unsigned)((nr + 255) / 256), 256, 0, st>>>(ra);
    CK(cudaGetLastError());
    k_env_center<<<(2 * n + 127) / 128, 128, 0, st>>>(Xv, nws, 2 * n, mv);
    k_env_center<<<(n + 127) / 128, 128, 0, st>>>(Xp, nws, n, mp);
    CK(cudaGetLastError());
    e2e_status s = truncated_svd(w, Xv, nws, 2 * n, r, Cv, Mv, sv + (int64_t)t * r, st, &full_svds);
    if (s != E2E_OK) return s;
    s = truncated_svd(w, Xp, nws, n, r, Cp, Mp, sv + (int64_t)(nt + t) * r, st, &full_svds);
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
    stats->transposed_vel = 2 * n < nws ? 1 : 0;
    stats->transposed_phi = n < nws ? 1 : 0;
    stats->full_svds = full_svds;
  }
  return E2E_OK;
}
