/*
 * ORACLE -- test infrastructure only.
 *
 * A plain-C, CPU restatement of the reference's Monte-Carlo transition builder
 * (rohit1607/e2e_GPU_DP, src/build_model.cu) and of its sparse value
 * iteration (src/spvi_2.cu), used as the parity checker for the CUDA path and
 * as the timed CPU baseline.  Only tests/, __graft_entry__.smoke() and the
 * cpu-baseline leg of bench.py load it; the product never links or calls it.
 *
 * Parity pinning: this restatement is checked against outputs of the
 * reference itself, compiled from its own sources for sm_100a (oracle/_ref)
 * and run on seeded inputs; those outputs are committed as fixtures under
 * tests/golden/ together with the script that made them.
 *
 * Floating point: every expression below is written in the order the
 * reference writes it, in float, with fmaf() exactly where nvcc's default
 * contraction (-fmad=true) fuses a product into the following add.  Build
 * with -ffp-contract=off so that the host compiler adds no fusions of its own.
 * The per-action cosf/sinf values are inputs (the reference evaluates them on
 * the device; passing the device's values keeps the comparison exact).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int32_t gsize, nt, nrzns, nmodes, num_actions;
  int32_t reward_type, i_term, j_term, term_subgrid_size, neighb_gsize;
  float dt, r_outbound, r_terminal, alpha;
} orc_problem;

typedef struct {
  const float *u, *v, *ui, *vi, *Yi, *s;
  const int32_t* mask;
} orc_fields;

typedef struct {
  const float *speed, *cosv, *sinv;
} orc_actions;

typedef struct {
  const orc_problem* P;
  const orc_fields* F;
  const float *xs, *ys;
  const orc_actions* A;
} orc_ctx;

/* ---- per-sample helpers --------------------------------------------------- */

/* is_terminal, src/build_model.cu:181-190 */
static int orc_is_terminal(const orc_problem* P, int i, int j) {
  return (i >= P->i_term && i < P->i_term + P->term_subgrid_size) &&
         (j >= P->j_term && j < P->j_term + P->term_subgrid_size);
}

/* is_in_obstacle, src/build_model.cu:172-178 (mask value must equal 1) */
static int orc_in_obstacle(const orc_ctx* c, int64_t sp, int T) {
  int64_t nc = (int64_t)c->P->gsize * c->P->gsize;
  return c->F->mask[(int64_t)T * nc + sp] == 1;
}

/* calculate_one_step_reward, src/build_model.cu:231-265 */
static float orc_step_reward(const orc_problem* P, float ac_speed, float rad1, float rad2) {
  const float Cr = 1.0f, Cf = 1.0f, Ct = 0.01f;
  float dt = P->dt;
  switch (P->reward_type) {
    case 0:
      return -dt;
    case 1:
      return -fmaf(Cf * ac_speed, ac_speed, Ct) * dt;
    case 2: {
      float a = (Cr * (rad2 + rad1)) / 2.0f;
      return (fmaf(-(Cf * ac_speed), ac_speed, a) - Ct) * dt;
    }
    case 3:
      return ((Cr * (rad2 + rad1)) / 2.0f - Ct) * dt;
    case 4: {
      float energy_reward = -(ac_speed * ac_speed) * dt;
      float time_reward = -dt;
      return fmaf(P->alpha, energy_reward, (1.0f - P->alpha) * time_reward);
    }
    default:
      return 0.0f;
  }
}

/* is_within_band, src/build_model.cu:419-441 */
static int orc_within_band(const orc_ctx* c, int i, int j, int i1, int j1, int i2, int j2) {
  if (i1 == i2 || j1 == j2) return 1;
  const float* xs = c->xs;
  const float* ys = c->ys;
  int g = c->P->gsize;
  float cell_diag = (float)((double)fabsf(xs[1] - xs[0]) * 1.414213);
  float x = xs[j], y = ys[g - 1 - i];
  float x1 = xs[j1], y1 = ys[g - 1 - i1];
  float x2 = xs[j2], y2 = ys[g - 1 - i2];
  float A = (y2 - y1) / (x2 - x1);
  float B = -1.0f;
  float C = fmaf(-A, x1, y1);
  float dist = fabsf(fmaf(A, x, B * y) + C) / sqrtf(fmaf(A, A, B * B));
  return dist < cell_diag;
}

/* goes_through_obstacle, src/build_model.cu:444-477 */
static int orc_through_obstacle(const orc_ctx* c, int i1, int j1, int i2, int j2, int T) {
  int g = c->P->gsize;
  int imin = i1 < i2 ? i1 : i2, imax = i1 < i2 ? i2 : i1;
  int jmin = j1 < j2 ? j1 : j2, jmax = j1 < j2 ? j2 : j1;
  for (int i = imin; i <= imax; i++)
    for (int j = jmin; j <= jmax; j++) {
      if (i == i1 && j == j1) continue;
      int64_t sp = (int64_t)j + (int64_t)g * i;
      if (orc_in_obstacle(c, sp, T) || orc_in_obstacle(c, sp, T + 1))
        if (orc_within_band(c, i, j, i1, j1, i2, j2)) return 1;
    }
  return 0;
}

/*
 * One sample (one reference thread of transition_calc, src/build_model.cu:483-559):
 * velocity (extract_velocity :361-404), move (:268-356), step reward, obstacle
 * override.  Returns the next cell and the reward; *near_edge is set when the
 * snapped coordinate lies within 1e-6 of a cell edge or a clamp bound.
 */
static void orc_sample(const orc_ctx* c, int T, int i1, int j1, int a, int rzn, int* i2o,
                       int* j2o, float* ro, int* near_edge) {
  const orc_problem* P = c->P;
  const orc_fields* Fd = c->F;
  const float* xs = c->xs;
  const float* ys = c->ys;
  int g = P->gsize, nm = P->nmodes;
  int64_t nc = (int64_t)g * g;
  int64_t sp = (int64_t)i1 * g + j1;
  int64_t mean_id = (int64_t)T * nc + sp;
  int64_t sp_uvi = (int64_t)T * nm * nc + (int64_t)g * i1 + j1;
  int64_t sp_Yi = (int64_t)T * P->nrzns * nm + (int64_t)rzn * nm;
  float sum_x = 0.0f, sum_y = 0.0f;
  for (int k = 0; k < nm; k++) sum_x = fmaf(Fd->ui[sp_uvi + k * nc], Fd->Yi[sp_Yi + k], sum_x);
  for (int k = 0; k < nm; k++) sum_y = fmaf(Fd->vi[sp_uvi + k * nc], Fd->Yi[sp_Yi + k], sum_y);
  float vx = Fd->u[mean_id] + sum_x;
  float vy = Fd->v[mean_id] + sum_y;
  float rad1 = Fd->s[mean_id];
  int i = i1, j = j1;
  float r = 0.0f;
  *near_edge = 0;
  if (!orc_is_terminal(P, i1, j1)) {
    if (!orc_in_obstacle(c, sp, T)) {
      /* move() */
      int n = g - 1;
      float F = c->A->speed[a];
      float dt = P->dt, r_out = P->r_outbound;
      float Dj = fabsf(xs[1] - xs[0]);
      float Di = fabsf(ys[1] - ys[0]);
      float vnetx = fmaf(F, c->A->cosv[a], vx);
      float vnety = fmaf(F, c->A->sinv[a], vy);
      float x = xs[j1], y = ys[g - 1 - i1];
      float xnew = fmaf(vnetx, dt, x);
      float ynew = fmaf(vnety, dt, y);
      if (fabsf(xnew - xs[n]) < 1e-6f || fabsf(xnew - xs[0]) < 1e-6f ||
          fabsf(ynew - ys[n]) < 1e-6f || fabsf(ynew - ys[0]) < 1e-6f)
        *near_edge = 1;
      if (xnew > xs[n]) {
        xnew = xs[n];
        r += r_out;
      } else if (xnew < xs[0]) {
        xnew = xs[0];
        r += r_out;
      }
      if (ynew > ys[n]) {
        ynew = ys[n];
        r += r_out;
      } else if (ynew < ys[0]) {
        ynew = ys[0];
        r += r_out;
      }
      float ax = xnew - xs[0];
      float ay = -(ynew - ys[n]);
      float remx = remainderf(ax, Dj);
      float remy = remainderf(ay, Di);
      int xind = (int)((ax - remx) / Dj);
      int yind = (int)((ay - remy) / Di);
      if (fabs(fabs((double)remx) - 0.5 * Dj) < 1e-6 || fabs(fabs((double)remy) - 0.5 * Di) < 1e-6)
        *near_edge = 1;
      if ((double)remx >= 0.5 * (double)Dj) xind += 1;
      if ((double)remy >= 0.5 * (double)Di) yind += 1;
      i = yind;
      j = xind;
      if (i == 0 || i == n || j == 0 || j == n) r += r_out;
      if (orc_is_terminal(P, i, j))
        r += P->r_terminal;
      else if (T > P->nt - 20)
        r = (float)fma(0.05, (double)r_out, (double)r);
      /* end of move() */
      int64_t sp2 = (int64_t)i * g + j;
      float rad2 = Fd->s[(int64_t)(T + 1) * nc + sp2];
      float r_step = orc_step_reward(P, F, rad1, rad2);
      r = r + r_step;
      if (orc_through_obstacle(c, i1, j1, i, j, T)) r = r_out;
    } else {
      r = P->r_outbound;
    }
  }
  *i2o = i;
  *j2o = j;
  *ro = r;
}

/* ---- public: single samples ---------------------------------------------- */

void orc_samples(const orc_problem* P, const orc_fields* F, const float* xs, const float* ys,
                 const float* speed, const float* cosv, const float* sinv, int T, int cell, int a,
                 int32_t* i2, int32_t* j2, float* r, int32_t* near_edge) {
  orc_actions A = {speed, cosv, sinv};
  orc_ctx c = {P, F, xs, ys, &A};
  int g = P->gsize;
  for (int rz = 0; rz < P->nrzns; rz++) {
    int ii, jj, ne;
    float rr;
    orc_sample(&c, T, cell / g, cell % g, a, rz, &ii, &jj, &rr, &ne);
    i2[rz] = ii;
    j2[rz] = jj;
    r[rz] = rr;
    near_edge[rz] = ne;
  }
}

/* ---- public: rows of the transition model --------------------------------- */

typedef struct {
  int64_t n_rows;
  int64_t nnz;
  int64_t* row_ptr; /* n_rows + 1 */
  int64_t* col;     /* absolute S2 */
  uint32_t* cnt;
  float* R;         /* one per row: sumR / nrzns */
  uint64_t dropped;     /* samples outside the m*m window (reference bin m*m or mis-binned) */
  uint64_t misbinned;   /* subset of dropped that the reference would write to a wrong bin */
  uint64_t near_edge;   /* samples within 1e-6 of a cell edge or clamp bound */
} orc_rows;

typedef struct {
  const orc_ctx* c;
  int64_t r0, r1;
  int64_t cap, nnz;
  int64_t* col;
  uint32_t* cnt;
  int64_t* rowlen;
  float* R;
  uint64_t dropped, misbinned, near_edge;
  int failed;
} orc_job;

static void* orc_rows_worker(void* arg) {
  orc_job* jb = (orc_job*)arg;
  const orc_ctx* c = jb->c;
  const orc_problem* P = c->P;
  int g = P->gsize, Na = P->num_actions, m = P->neighb_gsize, del = (m - 1) / 2;
  int64_t nc = (int64_t)g * g;
  uint32_t* hist = (uint32_t*)calloc((size_t)m * m, sizeof(uint32_t));
  if (!hist) {
    jb->failed = 1;
    return NULL;
  }
  for (int64_t row = jb->r0; row < jb->r1; row++) {
    int64_t s = row / Na;
    int a = (int)(row % Na);
    int T = (int)(s / nc);
    int64_t cell = s % nc;
    int i1 = (int)(cell / g), j1 = (int)(cell % g);
    memset(hist, 0, sizeof(uint32_t) * m * m);
    float sumR = 0.0f;
    for (int rz = 0; rz < P->nrzns; rz++) {
      int i2, j2, ne;
      float r;
      orc_sample(c, T, i1, j1, a, rz, &i2, &j2, &r, &ne);
      jb->near_edge += (uint64_t)ne;
      /* get_posids_relS2_0 / get_rel_sp_id2, src/build_model.cu:114-141 */
      int di = i2 - (i1 - del), dj = j2 - (j1 - del);
      if (di >= 0 && di < m && dj >= 0 && dj < m) {
        hist[dj + m * di] += 1u;
      } else {
        jb->dropped++;
        if (di < m && dj < m) jb->misbinned++;
      }
      sumR += r; /* atomicAdd(&sumR_sa[sp_id], r), :553 */
    }
    /* compute_mean, :563-570 */
    jb->R[row - jb->r0] = sumR / (float)P->nrzns;
    /* count_kernel + reduce_kernel, :574-644: nonzero bins in bin order */
    int64_t len = 0;
    for (int b = 0; b < m * m; b++) {
      if (!hist[b]) continue;
      if (jb->nnz >= jb->cap) {
        int64_t ncap = jb->cap * 2 + 1024;
        int64_t* nc2 = (int64_t*)realloc(jb->col, sizeof(int64_t) * ncap);
        uint32_t* nn2 = (uint32_t*)realloc(jb->cnt, sizeof(uint32_t) * ncap);
        if (nc2) jb->col = nc2;
        if (nn2) jb->cnt = nn2;
        if (!nc2 || !nn2) {
          jb->failed = 1;
          free(hist);
          return NULL;
        }
        jb->cap = ncap;
      }
      int i2 = b / m + (i1 - del), j2 = b % m + (j1 - del);
      jb->col[jb->nnz] = (int64_t)(T + 1) * nc + (int64_t)i2 * g + j2;
      jb->cnt[jb->nnz] = hist[b];
      jb->nnz++;
      len++;
    }
    jb->rowlen[row - jb->r0] = len;
  }
  free(hist);
  return NULL;
}

/*
 * Rows [r0, r1) of the model in state-major order: row = s*Na + a with
 * s = t*ncells + cell, t in [0, nt-1).  Entries of a row are the non-empty
 * neighbourhood bins in bin order, i.e. ascending S2 (the order of
 * reduce_kernel).  Returns 0 on success.
 */
int orc_build_rows(const orc_problem* P, const orc_fields* F, const float* xs, const float* ys,
                   const float* speed, const float* cosv, const float* sinv, int64_t r0,
                   int64_t r1, int nthreads, orc_rows* out) {
  memset(out, 0, sizeof(*out));
  if (r1 < r0 || nthreads < 1) return 1;
  orc_actions A = {speed, cosv, sinv};
  orc_ctx c = {P, F, xs, ys, &A};
  int64_t nrows = r1 - r0;
  if ((int64_t)nthreads > nrows && nrows > 0) nthreads = (int)nrows;
  if (nrows == 0) nthreads = 1;
  orc_job* jobs = (orc_job*)calloc((size_t)nthreads, sizeof(orc_job));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  int64_t* rowlen = (int64_t*)calloc((size_t)nrows + 1, sizeof(int64_t));
  out->R = (float*)calloc((size_t)nrows + 1, sizeof(float));
  if (!jobs || !th || !rowlen || !out->R) return 2;
  for (int k = 0; k < nthreads; k++) {
    jobs[k].c = &c;
    jobs[k].r0 = r0 + nrows * k / nthreads;
    jobs[k].r1 = r0 + nrows * (k + 1) / nthreads;
    jobs[k].cap = 0;
    jobs[k].rowlen = rowlen + (jobs[k].r0 - r0);
    jobs[k].R = out->R + (jobs[k].r0 - r0);
  }
  for (int k = 1; k < nthreads; k++) pthread_create(&th[k], NULL, orc_rows_worker, &jobs[k]);
  orc_rows_worker(&jobs[0]);
  for (int k = 1; k < nthreads; k++) pthread_join(th[k], NULL);
  int64_t nnz = 0;
  int failed = 0;
  for (int k = 0; k < nthreads; k++) {
    nnz += jobs[k].nnz;
    failed |= jobs[k].failed;
    out->dropped += jobs[k].dropped;
    out->misbinned += jobs[k].misbinned;
    out->near_edge += jobs[k].near_edge;
  }
  out->n_rows = nrows;
  out->nnz = nnz;
  out->row_ptr = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nrows + 1));
  out->col = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nnz + 1));
  out->cnt = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(nnz + 1));
  if (!failed && out->row_ptr && out->col && out->cnt) {
    out->row_ptr[0] = 0;
    for (int64_t r = 0; r < nrows; r++) out->row_ptr[r + 1] = out->row_ptr[r] + rowlen[r];
    int64_t off = 0;
    for (int k = 0; k < nthreads; k++) {
      if (jobs[k].nnz) {
        memcpy(out->col + off, jobs[k].col, sizeof(int64_t) * (size_t)jobs[k].nnz);
        memcpy(out->cnt + off, jobs[k].cnt, sizeof(uint32_t) * (size_t)jobs[k].nnz);
      }
      off += jobs[k].nnz;
    }
  } else {
    failed = 1;
  }
  for (int k = 0; k < nthreads; k++) {
    free(jobs[k].col);
    free(jobs[k].cnt);
  }
  free(jobs);
  free(th);
  free(rowlen);
  return failed ? 3 : 0;
}

void orc_rows_free(orc_rows* o) {
  free(o->row_ptr);
  free(o->col);
  free(o->cnt);
  free(o->R);
  memset(o, 0, sizeof(*o));
}

/* Host cosf/sinf of the action angles (CPU-only use; the device values are
 * passed instead whenever a GPU result is being compared). */
void orc_action_trig(const float* angle, int n, float* cosv, float* sinv) {
  for (int k = 0; k < n; k++) {
    cosv[k] = cosf(angle[k]);
    sinv[k] = sinf(angle[k]);
  }
}

/* ---- public: value iteration ------------------------------------------------ */

/*
 * Backup of one state s (select_best_action, src/spvi_2.cu:93-122, on the row
 * sums of Q = R + P V from solver_do_backup :174-260): max over actions with
 * the reference's start value -1e6 / action -1 and strict '>' (first max wins).
 * Rows exist for s < n_row_states; later states have Q = R only.
 */
static void orc_backup_f64(int64_t s, int Na, int64_t n_row_states, const int64_t* row_ptr,
                           const int64_t* col, const uint32_t* cnt, const float* val,
                           double inv_scale, const float* R, const double* Vin, double* vout,
                           int32_t* pout) {
  double best = -1e6;
  int32_t arg = -1;
  for (int a = 0; a < Na; a++) {
    int64_t row = s * Na + a;
    double q = (double)R[row];
    if (s < n_row_states) {
      double acc = 0.0;
      for (int64_t k = row_ptr[row]; k < row_ptr[row + 1]; k++) {
        double p = cnt ? (double)cnt[k] * inv_scale : (double)val[k];
        acc += p * Vin[col[k]];
      }
      q += acc;
    }
    if (q > best) {
      best = q;
      arg = a;
    }
  }
  *vout = best;
  *pout = arg;
}

/*
 * FP64 value iteration over a state-major CSR model (rows s*Na+a for
 * s < n_row_states).  mode 0: Jacobi from V = 0 until max|V'-V| < thresh
 * (solver_spvi_solve, src/spvi_2.cu:650-698) or max_iter sweeps; mode 1: one
 * Gauss-Seidel sweep in descending state order, which is backward induction
 * when every transition leads to a higher state index (the time-layered model
 * of src/build_model.cu:635).  Returns the number of sweeps; *resid gets the
 * last sup-norm (mode 0).
 */
int orc_vi_f64(int64_t Ns, int Na, int64_t n_row_states, const int64_t* row_ptr,
               const int64_t* col, const uint32_t* cnt, const float* val, double scale,
               const float* R, int mode, double thresh, int max_iter, double* V, int32_t* pi,
               double* resid) {
  double inv = scale > 0 ? 1.0 / scale : 1.0;
  if (mode == 1) {
    for (int64_t s = Ns - 1; s >= 0; s--) {
      double vo;
      int32_t po;
      orc_backup_f64(s, Na, n_row_states, row_ptr, col, cnt, val, inv, R, V, &vo, &po);
      V[s] = vo;
      pi[s] = po;
    }
    if (resid) *resid = 0.0;
    return 1;
  }
  double* W = (double*)calloc((size_t)Ns, sizeof(double));
  if (!W) return -1;
  for (int64_t s = 0; s < Ns; s++) V[s] = 0.0;
  int it = 0;
  double sup = 0.0;
  while (it < max_iter) {
    it++;
    sup = 0.0;
    for (int64_t s = 0; s < Ns; s++) {
      orc_backup_f64(s, Na, n_row_states, row_ptr, col, cnt, val, inv, R, V, &W[s], &pi[s]);
      double d = fabs(W[s] - V[s]);
      if (d > sup) sup = d;
    }
    memcpy(V, W, sizeof(double) * (size_t)Ns);
    if (sup < thresh) break;
  }
  free(W);
  if (resid) *resid = sup;
  return it;
}

/*
 * FP32 value iteration with the reference's float semantics: Q = R + sum of
 * (cnt/nrzns as float) * V in row order, argmax as above, float sup-norm,
 * stop when sup < thresh.  Returns the number of iterations.
 */
int orc_vi_f32(int64_t Ns, int Na, int64_t n_row_states, const int64_t* row_ptr,
               const int64_t* col, const uint32_t* cnt, const float* val, int32_t nrzns,
               const float* R, float thresh, int max_iter, float* V, int32_t* pi, float* resid) {
  float* W = (float*)calloc((size_t)Ns, sizeof(float));
  if (!W) return -1;
  for (int64_t s = 0; s < Ns; s++) V[s] = 0.0f;
  int it = 0;
  float sup = 0.0f;
  while (it < max_iter) {
    it++;
    sup = 0.0f;
    for (int64_t s = 0; s < Ns; s++) {
      float best = -1e6f;
      int32_t arg = -1;
      for (int a = 0; a < Na; a++) {
        int64_t row = s * Na + a;
        float q = R[row];
        if (s < n_row_states)
          for (int64_t k = row_ptr[row]; k < row_ptr[row + 1]; k++) {
            float p = cnt ? (float)cnt[k] / (float)nrzns : val[k];
            q = fmaf(p, V[col[k]], q);
          }
        if (q > best) {
          best = q;
          arg = a;
        }
      }
      W[s] = best;
      pi[s] = arg;
      float d = fabsf(W[s] - V[s]);
      if (d > sup) sup = d;
    }
    memcpy(V, W, sizeof(float) * (size_t)Ns);
    if (sup < thresh) break;
  }
  free(W);
  if (resid) *resid = sup;
  return it;
}

/*
 * FP64 backward induction over a large time-layered state-major CSR model, as
 * the library keeps it (int32 next states, integer counts scaled by 1/nrzns):
 * the same backup as orc_backup_f64 (first maximum from -1e6/-1, the rule of
 * src/spvi_2.cu:101-116), layer by layer from the last, the states of one
 * layer split over nthreads threads (they read only the next layer's values).
 * If pol is given, gap[s] = best Q(s, .) - Q(s, pol[s]) in FP64 (the margin by
 * which a given policy's action falls short of the best; pol[s] < 0 or >= Na
 * gives +inf).  Rows exist for states below (nt-1)*ncells; the last layer has
 * Q = R only.  Returns 0, or -1 if a thread could not be started.
 */
typedef struct {
  int64_t s0, s1;
  int Na;
  int64_t n_row_states;
  const int64_t* row_ptr;
  const int32_t* col;
  const uint32_t* cnt;
  const uint16_t* cnt16;
  double inv;
  const float* R;
  const int32_t* pol;
  double* V;
  int32_t* pi;
  double* gap;
} orc_layer_job;

static void* orc_layer_worker(void* arg) {
  const orc_layer_job* J = (const orc_layer_job*)arg;
  for (int64_t s = J->s0; s < J->s1; s++) {
    double best = -1e6, qpol = -INFINITY;
    int32_t arg_best = -1;
    const int32_t want = J->pol ? J->pol[s] : -1;
    for (int a = 0; a < J->Na; a++) {
      const int64_t row = s * J->Na + a;
      double q = (double)J->R[row];
      if (s < J->n_row_states) {
        double acc = 0.0;
        for (int64_t k = J->row_ptr[row]; k < J->row_ptr[row + 1]; k++) {
          const double c = J->cnt16 ? (double)J->cnt16[k] : (double)J->cnt[k];
          acc += c * J->inv * J->V[J->col[k]];
        }
        q += acc;
      }
      if (a == want) qpol = q;
      if (q > best) {
        best = q;
        arg_best = a;
      }
    }
    J->V[s] = best;
    J->pi[s] = arg_best;
    if (J->gap) J->gap[s] = (want >= 0 && want < J->Na) ? best - qpol : INFINITY;
  }
  return NULL;
}

int orc_vi_f64_layers(int64_t ncells, int nt, int Na, const int64_t* row_ptr, const int32_t* col,
                      const uint32_t* cnt, const uint16_t* cnt16, double scale, const float* R,
                      const int32_t* pol, int nthreads, double* V, int32_t* pi, double* gap) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  orc_layer_job jobs[256];
  const int64_t n_row_states = (int64_t)(nt - 1) * ncells;
  for (int t = nt - 1; t >= 0; t--) {
    const int64_t a0 = (int64_t)t * ncells, a1 = a0 + ncells;
    const int64_t per = (ncells + nthreads - 1) / nthreads;
    int started = 0;
    for (int k = 0; k < nthreads; k++) {
      orc_layer_job* J = &jobs[k];
      J->s0 = a0 + k * per;
      J->s1 = J->s0 + per < a1 ? J->s0 + per : a1;
      if (J->s0 > a1) J->s0 = a1;
      J->Na = Na;
      J->n_row_states = n_row_states;
      J->row_ptr = row_ptr;
      J->col = col;
      J->cnt = cnt;
      J->cnt16 = cnt16;
      J->inv = 1.0 / scale;
      J->R = R;
      J->pol = pol;
      J->V = V;
      J->pi = pi;
      J->gap = gap;
    }
    for (int k = 1; k < nthreads; k++) {
      if (pthread_create(&th[k], NULL, orc_layer_worker, &jobs[k]) != 0) {
        for (int j = 1; j < k; j++) pthread_join(th[j], NULL);
        return -1;
      }
      started = k;
    }
    orc_layer_worker(&jobs[0]);
    for (int k = 1; k <= started; k++) pthread_join(th[k], NULL);
  }
  return 0;
}
