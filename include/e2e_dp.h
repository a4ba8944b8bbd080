/*
 * e2e_dp.h -- C ABI of the B200 end-to-end dynamic-programming planner:
 * Monte-Carlo transition build -> CSR assembly -> sparse value iteration.
 *
 * The reference (rohit1607/e2e_GPU_DP) has no library API: its boundary is two
 * executables, src/build_model.cu (main :926) and src/spvi_2.cu (main :730),
 * that exchange .npy files.  Each entry point below names the reference
 * function or file-protocol step it replaces.  The drop-in executables
 * `build_model` and `spvi_2` of this package are thin C++ mains over this ABI
 * that keep the reference's command line and file layout.
 *
 * Conventions
 *  - Plain C types only; every function returns an e2e_status and never aborts.
 *  - `stream` is a cudaStream_t passed as void* (NULL = the legacy default stream).
 *  - `where` arguments say whether a pointer is host (E2E_HOST) or device (E2E_DEVICE)
 *    memory of the current CUDA device.
 *  - A model handle is owned by the caller and released with e2e_model_free().
 *    Handles are independent (no global state), so different host threads may
 *    work on different handles; one handle must not be used by two threads at once.
 *  - Indices: state s = t*ncells + i*gsize + j (src/build_model.cu:81-91); model row
 *    (s, a) has index s*num_actions + a ("state-major").  The reference's on-disk COO
 *    is action-major (row a*Ns + s); e2e_model_write_npy/e2e_model_read_npy convert.
 */
#ifndef E2E_DP_H
#define E2E_DP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define E2E_DP_ABI_VERSION 2

typedef enum {
  E2E_OK = 0,
  E2E_ERR_INVALID = 1,       /* bad argument or problem definition */
  E2E_ERR_CUDA = 2,          /* a CUDA runtime call failed (see e2e_last_error) */
  E2E_ERR_NOMEM = 3,         /* device or host allocation failed */
  E2E_ERR_IO = 4,            /* .npy read/write failed or a file is malformed */
  E2E_ERR_TIMEOUT = 5,       /* host wall-clock limit reached */
  E2E_ERR_NOT_CONVERGED = 6, /* max_iter reached before the threshold */
  E2E_ERR_UNSUPPORTED = 7,   /* valid input outside what this build implements */
  E2E_ERR_DEVICE = 8,        /* a device-side check failed (bounded wait, pool, overflow) */
  E2E_ERR_CANCELLED = 9,     /* request cancelled (server) */
  E2E_ERR_BUSY = 10          /* admission refused: not enough free device memory (server) */
} e2e_status;

enum { E2E_HOST = 0, E2E_DEVICE = 1 };

/* Count storage of a model: exact integer counts scaled by 1/nrzns, or plain
 * float probabilities (models read from arbitrary COO files). */
enum { E2E_COUNT_U16 = 0, E2E_COUNT_U32 = 1, E2E_VALUE_F32 = 2, E2E_COUNT_AUTO = -1 };

/*
 * Problem definition.  Fields 0..19 are the slots of the reference's 32-float
 * `prob_params` vector in slot order (src/build_model.cu:1032-1055, saved as
 * prob_params.npy at :1310); x0/y0 are the grid origin (header: x0 = dx/2,
 * src/input_to_build_model.h:14-15).  reward_type: 0 time, 1 energy1,
 * 2 energy2, 3 energy3, 4 custom1 (get_reward_type, src/build_model.cu:898-918).
 */
typedef struct {
  int32_t gsize;             /* 0 */
  int32_t num_actions;       /* 1 = num_ac_speeds * num_ac_angles */
  int32_t nrzns;             /* 2 */
  float F;                   /* 3 max vehicle speed */
  float dt;                  /* 4 */
  float r_outbound;          /* 5 */
  float r_terminal;          /* 6 */
  int32_t nmodes;            /* 7 */
  int32_t i_term;            /* 8 */
  int32_t j_term;            /* 9 */
  int32_t nt;                /* 10 */
  int32_t is_stationary;     /* 11 (unused by the kernels, as in the reference) */
  int32_t term_subgrid_size; /* 12 */
  int32_t reward_type;       /* 13 */
  int32_t num_ac_speeds;     /* 14 */
  int32_t num_ac_angles;     /* 15 */
  float dx;                  /* 16 */
  float dy;                  /* 17 */
  int32_t neighb_gsize;      /* 18 (m, odd, <= gsize) */
  float alpha;               /* 19 */
  float x0;                  /* grid origin, cell (.., j) centre x = x0 + j*dx */
  float y0;
} e2e_problem;

/*
 * Input fields in the reference's layout and dtypes (src/build_model.cu:978-1019):
 * u, v, s, mask: (nt, gsize, gsize); ui, vi: (nt, nmodes, gsize, gsize);
 * yi: (nt, nrzns, nmodes).  float32 except mask (int32; 1 = obstacle).
 */
typedef struct {
  const float* u;
  const float* v;
  const float* ui;
  const float* vi;
  const float* yi;
  const float* s;
  const int32_t* mask;
} e2e_fields;

typedef struct {
  int32_t count_type;   /* E2E_COUNT_AUTO (u16 when nrzns < 65536), E2E_COUNT_U16 or _U32 */
  int32_t tile_cells;   /* 0 = default (32); cells per builder tile, multiple of 32 */
  int64_t stage_hint;   /* 0 = default; initial staging capacity in entries */
  int32_t keep_reward_parts; /* 1: also keep each row's reward sum (before the division by nrzns),
                                which re-targeting a model needs (the request server) */
  int32_t reserved;
} e2e_build_opts;

typedef struct {
  int64_t ns;            /* states = nt * gsize^2 */
  int64_t n_rows;        /* rows with transitions = (nt-1) * gsize^2 * num_actions */
  int64_t nnz;
  int32_t num_actions;
  int32_t nt;
  int32_t ncells;
  int32_t nrzns;         /* count scale (1 for E2E_VALUE_F32 models) */
  int32_t count_type;    /* E2E_COUNT_U16, _U32 or E2E_VALUE_F32 */
  int32_t index_bits;    /* 32 or 64: width of row_ptr */
  const void* row_ptr;   /* device, n_rows + 1 (int32 or int64) */
  const int32_t* col;    /* device, nnz: absolute next state S2 */
  const void* cnt;       /* device, nnz: uint16 / uint32 counts or float values */
  const float* R;        /* device, ns * num_actions, state-major */
  uint64_t dropped;      /* samples outside the m x m neighbourhood (not counted, as the reference's bin m*m) */
  uint64_t overflow_units; /* rows whose samples spread beyond the builder's fast window */
  double build_kernel_ms;  /* device time of the last builder launch (CUDA events on the build stream) */
  double assemble_ms;      /* device time of the CSR assembly (tile scan + copy) */
  int32_t build_launches;  /* builder launches (1, or 2 after a re-run with larger buffers) */
  int32_t reserved;
} e2e_model_info;

typedef struct e2e_model e2e_model;

typedef struct {
  int32_t method;        /* 0 = Jacobi sweeps from V=0 (reference semantics),
                            1 = layered backward sweep + one verification sweep */
  float threshold;       /* Jacobi stop: sup-norm < threshold (reference default 0.1) */
  int32_t max_iter;      /* 0 = nt + 2 */
  double timeout_s;      /* host wall-clock limit, 0 = none */
  int32_t fp64_check;    /* 1: FP64 backward solve on the device, report the error of the FP32 values */
  int32_t schedule;      /* 0 = automatic.  Bits 0-3: warps sharing a 32-state chunk in the layered
                            sweep (0 = auto, 1, 2, 4, 8).  Bit 8 set: bits 4-7 give the sweep
                            tuning (4: L2 prefetch of the chunk a warp takes next, 5: of the chunk
                            it starts, 6: lean kernel without entry look-ahead, 7: Jacobi sweeps
                            staged through shared memory by TMA bulk copies). */
} e2e_vi_opts;

typedef struct {
  int32_t iterations;      /* sweeps performed (layered: 1 + verification sweep) */
  double residual;         /* last sup-norm |V' - V| (FP64 reduction) */
  double seconds;          /* device time of the solve (CUDA events) */
  double fp64_max_abs_err; /* fp64_check: max |V32 - V64| */
  double fp64_max_rel_err; /* fp64_check: max |V32 - V64| / max |V64| */
  int64_t bytes_per_sweep; /* algorithmic bytes of one sweep (CSR form: row_ptr, col, count, R, V) */
  int64_t stream_bytes_per_sweep; /* bytes a sweep over the sliced copy moves (padding included) */
  double pack_ms;          /* device time spent building the sliced copy in this call (0 if cached) */
  double sweep_seconds;    /* layered: device time of the backward pass alone */
} e2e_vi_stats;

/* ---- library ------------------------------------------------------------ */
int e2e_abi_version(void);
const char* e2e_status_string(e2e_status st);
/* Message of the last failure on the calling host thread ("" if none). */
const char* e2e_last_error(void);

/* Release the device memory the library keeps cached for later builds and
 * solves (its stream-ordered pool never returns memory on its own).  Waits for
 * the device.  No counterpart in the reference, whose thrust vectors allocate
 * and free per (t, a). */
e2e_status e2e_memory_trim(void);

/* prob_params.npy slots <-> e2e_problem (src/build_model.cu:1032-1055). */
e2e_status e2e_problem_from_params(const float prob_params[32], e2e_problem* out);
e2e_status e2e_problem_to_params(const e2e_problem* p, float prob_params_out[32]);

/* Action table: speed and heading per action index j + num_ac_angles*i
 * (populate_actions, src/build_model.cu:1438-1457) and their cosf/sinf as
 * evaluated on the device (the builder's move(), src/build_model.cu:284-285). */
e2e_status e2e_action_table(const e2e_problem* p, float* speed, float* angle, float* cosv,
                            float* sinv);

/* ---- build (replaces build_model main, src/build_model.cu:926-1238, and the
 * per-(t,a) worker build_sparse_transition_model_at_T_at_a, :696-892) --------
 * Limit the reference does not have: nrzns <= 32767 (a row's window counters
 * are 16 bits, bit 15 marking an obstacle-overridden bin); above it the call
 * returns E2E_ERR_UNSUPPORTED.  The same holds for e2e_build_solve. */
e2e_status e2e_build_model(const e2e_problem* p, const e2e_fields* fields, int fields_where,
                           const e2e_build_opts* opts /* may be NULL */, e2e_model** out,
                           void* stream);
e2e_status e2e_model_free(e2e_model* m);
e2e_status e2e_model_get_info(const e2e_model* m, e2e_model_info* info);

/* Copy the CSR to host buffers (any may be NULL): row_ptr as int64 (n_rows+1),
 * col (nnz), counts widened to uint32 (nnz; E2E_VALUE_F32 models: the float bits),
 * R (ns*num_actions). */
e2e_status e2e_model_copy_to_host(const e2e_model* m, int64_t* row_ptr, int32_t* col,
                                  uint32_t* cnt, float* R, void* stream);

/* Write the reference's model files into `dir` (save_master_Coos_to_file,
 * src/build_model.cu:1246-1314): master_cooS1/S2 (int64, or int32 after the
 * reference's convert step when index_bits == 32, src/convert_model_datatype.py:19-23),
 * master_cooVal (f32 count/nrzns), master_R (f32, action-major), DP_relv_params
 * (int64 [Ns, Na]) and prob_params (f32[32]). */
e2e_status e2e_model_write_npy(const e2e_model* m, const e2e_problem* p, const char* dir,
                               int index_bits);

/* Load a model directory in the reference layout (get_mdp_model,
 * src/spvi_2.cu:393-504): S1/S2 int32 or int64, Val f32, R f32, DP_relv_params.
 * If prob_params.npy is present and every value is count/nrzns, the model is
 * stored as exact counts; otherwise as float values. */
e2e_status e2e_model_read_npy(const char* dir, e2e_model** out, void* stream);

/* ---- solve (replaces solver_spvi_solve, src/spvi_2.cu:650-726, with the
 * backup of solver_do_backup :174-260, select_best_action :93-122 and
 * compute_sup_norm :263-356 fused into one kernel per sweep) ----------------- */
e2e_status e2e_spvi_solve(const e2e_model* m, const e2e_vi_opts* opts /* may be NULL */,
                          int32_t* policy_out, float* value_out, int out_where,
                          e2e_vi_stats* stats /* may be NULL */, void* stream);

/* ---- many layered solves in one launch ---------------------------------------
 * No counterpart in the reference, which solves one model per spvi_2 process.
 * Solves n time-layered models with the layered schedule in one persistent
 * cooperative launch (a grid barrier per layer step, models aligned on their
 * last layer), captured in a CUDA graph that later batches of the same launch
 * shape replay.  Results are bit-identical to e2e_spvi_solve(method = 1) on each
 * model.  value_dev[i] / policy_dev[i]: device buffers of model i's ns states.
 * opts->schedule as for e2e_spvi_solve, plus bit 9: launch directly, no graph,
 * and bit 10: pick the schedule by a rule (no timing runs); without bits 8 and
 * 10 the schedule (warps per chunk, kernel variant, L2 prefetch) is autotuned
 * on the first batch of each shape.
 * Calls are serialised inside the library. */
/* Builds n problems (problems[i] with fields[i], all in fields_where memory)
 * with e2e_build_model on `workers` host threads, each with its own stream
 * (0 = 4), so that small builds overlap on the device.  The models are the same
 * as one build at a time.  On failure every model is freed and out[] is NULL. */
e2e_status e2e_build_models(const e2e_problem* problems, const e2e_fields* fields, int32_t n,
                            int fields_where, const e2e_build_opts* opts /* may be NULL */,
                            int32_t workers, e2e_model** out);

typedef struct {
  int32_t jobs, launches;
  int32_t groups, tune, grid; /* schedule used: warps per chunk, tuning bits, CTAs */
  int32_t graph;              /* 1: replayed from a CUDA graph */
  double seconds;             /* device time of the launches (CUDA events) */
  double pack_ms;             /* sliced copies built by this call */
  double tune_ms;             /* autotuning spent in this call */
  int64_t stream_bytes;       /* bytes one pass over all the models' sliced copies moves */
} e2e_batch_stats;

e2e_status e2e_spvi_solve_batch(const e2e_model* const* models, int32_t n, const e2e_vi_opts* opts,
                                float* const* value_dev, int32_t* const* policy_dev,
                                e2e_batch_stats* stats /* may be NULL */, void* stream);

/* ---- request server (served form) ---------------------------------------------
 * No counterpart in the reference, which plans one problem per build_model +
 * spvi_2 run.  A server keeps velocity fields resident, builds one base model per
 * (field, heading set) on first use (no terminal cells, reward sums kept), and
 * answers plan requests by re-targeting R around each request's target and
 * solving all queued requests in one batched launch (continuous batching).  A
 * worker thread owns the device work; admission is by an HBM budget, evicting
 * idle models least recently used.  For integer-valued rewards (the "time"
 * reward with integer dt, r_outbound, r_terminal) results are bit-identical to
 * building the model with the request's target and calling e2e_spvi_solve;
 * otherwise they differ by the rounding of the reward sums.  The terminal
 * subgrid of a request is its target cell (term_subgrid_size 1). */
typedef struct e2e_server e2e_server;

typedef struct {
  int64_t hbm_budget;  /* bytes for models and requests; 0 = 80% of the free memory at creation */
  int32_t max_batch;   /* requests per launch; 0 = 256 (at most 1024) */
  int32_t schedule;    /* e2e_vi_opts.schedule of the batched launches (0 = rule-based, no timing runs) */
} e2e_server_opts;

typedef struct {
  int32_t field_id;      /* from e2e_server_add_field */
  int32_t num_ac_angles; /* heading set: this many headings j*2pi/n (speeds as the field's problem) */
  int32_t i_term, j_term; /* target cell */
  int32_t i_start, j_start; /* start cell (layer 0): its value and action are returned */
  int32_t keep_outputs;  /* 1: keep the full value and policy arrays for e2e_server_fetch */
  int32_t reserved;
  int64_t tag;           /* returned with the result */
} e2e_request;

typedef struct {
  int64_t request_id, tag;
  int32_t status;        /* E2E_OK or the failure */
  int32_t action_at_start;
  float value_at_start;
  int32_t batch_size;    /* requests solved in the same launch */
  double latency_ms;     /* submission to completion (host steady clock) */
  double queue_ms;       /* submission to being taken into a batch */
} e2e_result;

typedef struct {
  int64_t completed, failed, pending, batches;
  int64_t models_built, models_evicted, models_resident;
  int64_t bytes_in_use, budget_bytes;
  int32_t max_batch, reserved;
  double build_ms, solve_ms; /* host time building base models; device time of the batched launches */
} e2e_server_stats;

e2e_status e2e_server_create(const e2e_server_opts* opts /* may be NULL */, e2e_server** out);
/* p: grid, nt, nrzns, nmodes, speeds, dt, dx, dy, rewards of the field (its
 * target and heading count are ignored); fields as for e2e_build_model, copied. */
e2e_status e2e_server_add_field(e2e_server* s, const e2e_problem* p, const e2e_fields* f, int fields_where,
                                int32_t* field_id);
e2e_status e2e_server_submit(e2e_server* s, const e2e_request* r, int64_t* request_id);
/* Cancel a request that is still queued: its result (status E2E_ERR_CANCELLED)
 * is returned by e2e_server_poll.  E2E_ERR_BUSY if a batch has already taken it
 * (it completes normally), E2E_ERR_INVALID for an unknown id.  No counterpart in
 * the reference (whose solver declares a timeout status it never sets,
 * src/spvi_2.cu:650-726). */
e2e_status e2e_server_cancel(e2e_server* s, int64_t request_id);
/* up to max finished results; waits up to wait_s seconds when none is ready */
e2e_status e2e_server_poll(e2e_server* s, e2e_result* out, int32_t max, int32_t* n_out, double wait_s);
/* full value / policy (ns = nt * gsize^2 each) of a finished keep_outputs request */
e2e_status e2e_server_fetch(e2e_server* s, int64_t request_id, float* value_out, int32_t* policy_out,
                            int out_where);
e2e_status e2e_server_get_stats(e2e_server* s, e2e_server_stats* out);
e2e_status e2e_server_destroy(e2e_server* s);

/* ---- policy rollout evaluation ------------------------------------------------
 * Replaces the reference's Python trajectory loop (Post_processing/
 * plot_e2eGPU_policy.py:433-474, plot_exact_trajectory_set_DP without policy
 * interpolation, moving with Grid.move_exact, grid_world.py:160-271) and
 * get_metrics (:776-797): one GPU thread follows the policy from the start cell
 * for each realisation of the velocity field, on continuous positions, until
 * the target (terminal subgrid of p), an edge or obstacle cell, or the last
 * step.  Float32 arithmetic as the reference under NumPy's scalar rules; the
 * mode sum of the velocity is a sequential fma chain. */
enum { E2E_ROLLOUT_INTERP = 1 };
typedef struct {
  int32_t i_start, j_start; /* start cell at t = 0 */
  int32_t n_rzns;           /* realisations to follow (0 = all of the field's) */
  int32_t flags;            /* E2E_ROLLOUT_INTERP: actions after the first interpolated from the policy of
                               the four cells around the position (the script's with_policy_interp,
                               Post_processing/plot_e2eGPU_policy.py:174-198); 0: the cell's own action */
} e2e_rollout_opts;

typedef struct {
  int32_t n, successes, failures, undecided, invalid; /* invalid: the policy had no action there */
  int32_t reserved;
  double success_rate;
  double mean_time, mean_energy_cons, mean_energy_col, mean_net_energy; /* over successes */
  double seconds;           /* device time of the rollout kernel */
} e2e_rollout_stats;

/* policy: ns int32 (host or device); outputs (host, each may be NULL): success
 * int8 per realisation (1 target, 0 failed, -1 undecided, -2 invalid policy),
 * travel time int32, energies float32 x3 (sum F^2, sum mean scalar field, their
 * difference), final (t, i, j) int32 x3. */
e2e_status e2e_rollout(const e2e_problem* p, const e2e_fields* f, int fields_where, const int32_t* policy,
                       int policy_where, const e2e_rollout_opts* opts, int8_t* success_out, int32_t* time_out,
                       float* energy_out, int32_t* final_out, e2e_rollout_stats* stats, void* stream);

/* ---- build and solve in one backward pass ------------------------------------
 * No counterpart in the reference, which writes the model between build_model
 * and spvi_2.  Layers nt-2 down to 0: the rows of layer t are built exactly as
 * by e2e_build_model and backed up at once against the finished values of
 * layer t+1, so the transition model is never stored (device memory: the
 * fields, V and policy).  Value and policy are bit-identical to
 * e2e_build_model + e2e_spvi_solve with the layered method (whose fixed point
 * is the Jacobi one); last layer: value 0, action 0.  policy_out / value_out:
 * ns entries each in out_where memory (either may be NULL).  One cooperative
 * launch: a tile's backup waits (bounded by E2E_WAIT_LIMIT_MS, default 5000)
 * for the next layer's completion; a wait that runs out gives E2E_ERR_DEVICE. */
typedef struct {
  double seconds;          /* device time of the pass (CUDA events) */
  int64_t n_rows;          /* rows built and backed up */
  int64_t nnz;             /* entries backed up (the model's nnz) */
  uint64_t dropped;        /* as e2e_model_info */
  uint64_t misbinned;
  uint64_t overflow_rows;
  int32_t launches;        /* kernel launches (one cooperative launch per pass; a pass is re-run when rows needed more dense histograms) */
  int32_t reserved;
  int64_t h2d_bytes;       /* field bytes copied from host memory */
} e2e_fused_stats;

e2e_status e2e_build_solve(const e2e_problem* p, const e2e_fields* fields, int fields_where,
                           int32_t* policy_out, float* value_out, int out_where,
                           e2e_fused_stats* stats /* may be NULL */, void* stream);

/* ---- environment generator (replaces build_environment_DG_with_westward_clouds,
 * src/data_input/build_environment_DG_with_westward_clouds.py:510-590) --------
 * Double-gyre velocity realisations for n_wsamples frequencies w in w_range on
 * an init_gsize grid, per time step a rank-n_modes reduction of the centred
 * realisations (mean = all_u_mat/all_v_mat, modes = all_ui_mat/all_vi_mat,
 * coefficients = all_Yi; the same for the scalar field phi), interpolation of
 * means and modes to the init_gsize*interpolate_degree grid, the moving scalar
 * cloud (all_s_mat) and the obstacle mask.  The reference's scipy griddata
 * 'linear' is evaluated from a table the caller provides: per fine point
 * (row-major over the fine grid, as griddata's (xgrid, ygrid) points) the three
 * vertex indices of its Delaunay triangle over the coarse cell centres (-1: outside
 * the hull, value 0) and their barycentric weights, as scipy computes them
 * (e2e_gpu_dp_b200.envgen.interp_table builds it).  Modes are defined up to sign:
 * each mode's largest-magnitude coefficient is made positive (products of modes
 * and coefficients, which is all the builder reads, do not depend on it).
 * Outputs: nt x G x G (u, v, phi, s, mask), nt x n_modes x G x G (ui, vi, phi_i),
 * nt x n_wsamples x n_modes (yi, phi_yi); G = init_gsize * interpolate_degree. */
enum { E2E_OBST_NONE = 0, E2E_OBST_STATIC = 1, E2E_OBST_DYNAMIC = 2 };
typedef struct {
  int32_t init_gsize, nt, n_wsamples, n_modes, interpolate_degree;
  int32_t obstacle_mode;   /* E2E_OBST_*: fill_obstacles (:441-468) */
  double dt, dxy, A, A_sc, eps, w_lo, w_hi, wx;
  double obs_upper_row, obs_left_col, obs_width, obs_speed_x, obs_speed_y; /* dynamic obstacle */
} e2e_env_params;
typedef struct {
  float *u, *v, *ui, *vi, *yi, *phi, *phi_i, *phi_yi, *s;
  int32_t* mask;
} e2e_env_fields;
typedef struct {
  double seconds;          /* device time (CUDA events) */
  int32_t fine_gsize;
  int32_t transposed_vel;  /* always 0 (kept for the layout: no reduction transposes its matrix) */
  int32_t transposed_phi;  /* always 0 */
  int32_t full_svds;       /* reductions whose range finder was re-run enlarged before it certified */
} e2e_env_stats;
/* interp_vertices / interp_weights: (G*G) x 3, host or device memory.
 * svals_out (may be NULL): 2 x nt x n_modes singular values (velocity, then phi). */
e2e_status e2e_env_generate(const e2e_env_params* p, const int32_t* interp_vertices,
                            const double* interp_weights, int out_where, const e2e_env_fields* out,
                            double* svals_out, e2e_env_stats* stats /* may be NULL */, void* stream);

/* ---- solve without device allocation ----------------------------------------
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory (a serving loop whose memory is fully reserved by its own pool, or code
 * running while another framework's allocator owns the device).  Same sweeps
 * and results as e2e_spvi_solve, outputs in caller-provided DEVICE buffers; its
 * scratch is a fixed 32 MiB file-scope device array, so models above
 * 8,388,544 states (or fp64_check) are rejected with E2E_ERR_UNSUPPORTED; the
 * number of sweeps is not limited.  The first call on a device caches the
 * array's address (make it before any stream capture; do not call it again
 * after cudaDeviceReset); all calls share the array, so calls that overlap on
 * the GPU race.  The layered method reports the actions of its verification
 * sweep, the same as the layered pass's for every model the builder makes. */
e2e_status e2e_spvi_solve_noalloc(const e2e_model* m, const e2e_vi_opts* opts /* may be NULL */,
                                  int32_t* policy_dev, float* value_dev,
                                  e2e_vi_stats* stats /* may be NULL */, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* E2E_DP_H */
