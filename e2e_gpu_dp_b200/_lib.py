"""ctypes binding of the C ABI in include/e2e_dp.h (libe2edp.so, built in-tree).

The library is the only compute path: if it is missing the import fails
loudly; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libe2edp.so")

E2E_OK = 0
E2E_ERR_INVALID = 1
E2E_HOST, E2E_DEVICE = 0, 1
E2E_COUNT_U16, E2E_COUNT_U32, E2E_VALUE_F32, E2E_COUNT_AUTO = 0, 1, 2, -1

STATUS = {
    0: "E2E_OK", 1: "E2E_ERR_INVALID", 2: "E2E_ERR_CUDA", 3: "E2E_ERR_NOMEM", 4: "E2E_ERR_IO",
    5: "E2E_ERR_TIMEOUT", 6: "E2E_ERR_NOT_CONVERGED", 7: "E2E_ERR_UNSUPPORTED",
    8: "E2E_ERR_DEVICE", 9: "E2E_ERR_CANCELLED", 10: "E2E_ERR_BUSY",
}


class E2EError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class Problem(C.Structure):
    _fields_ = [
        ("gsize", C.c_int32), ("num_actions", C.c_int32), ("nrzns", C.c_int32), ("F", C.c_float),
        ("dt", C.c_float), ("r_outbound", C.c_float), ("r_terminal", C.c_float),
        ("nmodes", C.c_int32), ("i_term", C.c_int32), ("j_term", C.c_int32), ("nt", C.c_int32),
        ("is_stationary", C.c_int32), ("term_subgrid_size", C.c_int32),
        ("reward_type", C.c_int32), ("num_ac_speeds", C.c_int32), ("num_ac_angles", C.c_int32),
        ("dx", C.c_float), ("dy", C.c_float), ("neighb_gsize", C.c_int32), ("alpha", C.c_float),
        ("x0", C.c_float), ("y0", C.c_float),
    ]


class Fields(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("u", "v", "ui", "vi", "yi", "s", "mask")]


class BuildOpts(C.Structure):
    _fields_ = [("count_type", C.c_int32), ("tile_cells", C.c_int32), ("stage_hint", C.c_int64),
                ("keep_reward_parts", C.c_int32), ("reserved", C.c_int32)]


class ModelInfo(C.Structure):
    _fields_ = [
        ("ns", C.c_int64), ("n_rows", C.c_int64), ("nnz", C.c_int64), ("num_actions", C.c_int32),
        ("nt", C.c_int32), ("ncells", C.c_int32), ("nrzns", C.c_int32), ("count_type", C.c_int32),
        ("index_bits", C.c_int32), ("row_ptr", C.c_void_p), ("col", C.c_void_p),
        ("cnt", C.c_void_p), ("R", C.c_void_p), ("dropped", C.c_uint64),
        ("overflow_units", C.c_uint64), ("build_kernel_ms", C.c_double),
        ("assemble_ms", C.c_double), ("build_launches", C.c_int32), ("reserved", C.c_int32),
    ]


class ViOpts(C.Structure):
    _fields_ = [("method", C.c_int32), ("threshold", C.c_float), ("max_iter", C.c_int32),
                ("timeout_s", C.c_double), ("fp64_check", C.c_int32), ("schedule", C.c_int32)]


class ViStats(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("residual", C.c_double), ("seconds", C.c_double),
                ("fp64_max_abs_err", C.c_double), ("fp64_max_rel_err", C.c_double),
                ("bytes_per_sweep", C.c_int64), ("stream_bytes_per_sweep", C.c_int64),
                ("pack_ms", C.c_double), ("sweep_seconds", C.c_double)]


class BatchStats(C.Structure):
    _fields_ = [("jobs", C.c_int32), ("launches", C.c_int32), ("groups", C.c_int32),
                ("tune", C.c_int32), ("grid", C.c_int32), ("graph", C.c_int32),
                ("seconds", C.c_double), ("pack_ms", C.c_double), ("tune_ms", C.c_double),
                ("stream_bytes", C.c_int64)]


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget", C.c_int64), ("max_batch", C.c_int32), ("schedule", C.c_int32)]


class Request(C.Structure):
    _fields_ = [("field_id", C.c_int32), ("num_ac_angles", C.c_int32), ("i_term", C.c_int32),
                ("j_term", C.c_int32), ("i_start", C.c_int32), ("j_start", C.c_int32),
                ("keep_outputs", C.c_int32), ("reserved", C.c_int32), ("tag", C.c_int64)]


class Result(C.Structure):
    _fields_ = [("request_id", C.c_int64), ("tag", C.c_int64), ("status", C.c_int32),
                ("action_at_start", C.c_int32), ("value_at_start", C.c_float), ("batch_size", C.c_int32),
                ("latency_ms", C.c_double), ("queue_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_int64), ("failed", C.c_int64), ("pending", C.c_int64),
                ("batches", C.c_int64), ("models_built", C.c_int64), ("models_evicted", C.c_int64),
                ("models_resident", C.c_int64), ("bytes_in_use", C.c_int64), ("budget_bytes", C.c_int64),
                ("max_batch", C.c_int32), ("reserved", C.c_int32), ("build_ms", C.c_double),
                ("solve_ms", C.c_double)]


class RolloutOpts(C.Structure):
    _fields_ = [("i_start", C.c_int32), ("j_start", C.c_int32), ("n_rzns", C.c_int32), ("flags", C.c_int32)]


E2E_ROLLOUT_INTERP = 1


class RolloutStats(C.Structure):
    _fields_ = [("n", C.c_int32), ("successes", C.c_int32), ("failures", C.c_int32), ("undecided", C.c_int32),
                ("invalid", C.c_int32), ("reserved", C.c_int32), ("success_rate", C.c_double),
                ("mean_time", C.c_double), ("mean_energy_cons", C.c_double), ("mean_energy_col", C.c_double),
                ("mean_net_energy", C.c_double), ("seconds", C.c_double)]


class FusedStats(C.Structure):
    _fields_ = [("seconds", C.c_double), ("n_rows", C.c_int64), ("nnz", C.c_int64), ("dropped", C.c_uint64),
                ("misbinned", C.c_uint64), ("overflow_rows", C.c_uint64), ("launches", C.c_int32),
                ("reserved", C.c_int32), ("h2d_bytes", C.c_int64)]


E2E_OBST_NONE, E2E_OBST_STATIC, E2E_OBST_DYNAMIC = 0, 1, 2


class EnvParams(C.Structure):
    _fields_ = [("init_gsize", C.c_int32), ("nt", C.c_int32), ("n_wsamples", C.c_int32), ("n_modes", C.c_int32),
                ("interpolate_degree", C.c_int32), ("obstacle_mode", C.c_int32), ("dt", C.c_double),
                ("dxy", C.c_double), ("A", C.c_double), ("A_sc", C.c_double), ("eps", C.c_double),
                ("w_lo", C.c_double), ("w_hi", C.c_double), ("wx", C.c_double), ("obs_upper_row", C.c_double),
                ("obs_left_col", C.c_double), ("obs_width", C.c_double), ("obs_speed_x", C.c_double),
                ("obs_speed_y", C.c_double)]


class EnvFields(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("u", "v", "ui", "vi", "yi", "phi", "phi_i", "phi_yi", "s", "mask")]


class EnvStats(C.Structure):
    _fields_ = [("seconds", C.c_double), ("fine_gsize", C.c_int32), ("transposed_vel", C.c_int32),
                ("transposed_phi", C.c_int32), ("full_svds", C.c_int32)]


# every exported symbol of include/e2e_dp.h with its signature
SIGNATURES = {
    "e2e_abi_version": (C.c_int, []),
    "e2e_status_string": (C.c_char_p, [C.c_int]),
    "e2e_last_error": (C.c_char_p, []),
    "e2e_memory_trim": (C.c_int, []),
    "e2e_problem_from_params": (C.c_int, [C.POINTER(C.c_float), C.POINTER(Problem)]),
    "e2e_problem_to_params": (C.c_int, [C.POINTER(Problem), C.POINTER(C.c_float)]),
    "e2e_action_table": (C.c_int, [C.POINTER(Problem)] + [C.POINTER(C.c_float)] * 4),
    "e2e_build_model": (C.c_int, [C.POINTER(Problem), C.POINTER(Fields), C.c_int,
                                  C.POINTER(BuildOpts), C.POINTER(C.c_void_p), C.c_void_p]),
    "e2e_model_free": (C.c_int, [C.c_void_p]),
    "e2e_model_get_info": (C.c_int, [C.c_void_p, C.POINTER(ModelInfo)]),
    "e2e_model_copy_to_host": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]),
    "e2e_model_write_npy": (C.c_int, [C.c_void_p, C.POINTER(Problem), C.c_char_p, C.c_int]),
    "e2e_model_read_npy": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p), C.c_void_p]),
    "e2e_spvi_solve": (C.c_int, [C.c_void_p, C.POINTER(ViOpts), C.c_void_p, C.c_void_p, C.c_int,
                                 C.POINTER(ViStats), C.c_void_p]),
    "e2e_spvi_solve_noalloc": (C.c_int, [C.c_void_p, C.POINTER(ViOpts), C.c_void_p, C.c_void_p,
                                         C.POINTER(ViStats), C.c_void_p]),
    "e2e_spvi_solve_batch": (C.c_int, [C.POINTER(C.c_void_p), C.c_int32, C.POINTER(ViOpts),
                                       C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                       C.POINTER(BatchStats), C.c_void_p]),
    "e2e_build_models": (C.c_int, [C.POINTER(Problem), C.POINTER(Fields), C.c_int32, C.c_int,
                                   C.POINTER(BuildOpts), C.c_int32, C.POINTER(C.c_void_p)]),
    "e2e_rollout": (C.c_int, [C.POINTER(Problem), C.POINTER(Fields), C.c_int, C.c_void_p, C.c_int,
                              C.POINTER(RolloutOpts), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                              C.POINTER(RolloutStats), C.c_void_p]),
    "e2e_build_solve": (C.c_int, [C.POINTER(Problem), C.POINTER(Fields), C.c_int, C.c_void_p, C.c_void_p,
                                  C.c_int, C.POINTER(FusedStats), C.c_void_p]),
    "e2e_env_generate": (C.c_int, [C.POINTER(EnvParams), C.c_void_p, C.c_void_p, C.c_int, C.POINTER(EnvFields),
                                   C.c_void_p, C.POINTER(EnvStats), C.c_void_p]),
    "e2e_server_create": (C.c_int, [C.POINTER(ServerOpts), C.POINTER(C.c_void_p)]),
    "e2e_server_add_field": (C.c_int, [C.c_void_p, C.POINTER(Problem), C.POINTER(Fields), C.c_int,
                                       C.POINTER(C.c_int32)]),
    "e2e_server_submit": (C.c_int, [C.c_void_p, C.POINTER(Request), C.POINTER(C.c_int64)]),
    "e2e_server_cancel": (C.c_int, [C.c_void_p, C.c_int64]),
    "e2e_server_poll": (C.c_int, [C.c_void_p, C.POINTER(Result), C.c_int32, C.POINTER(C.c_int32),
                                  C.c_double]),
    "e2e_server_fetch": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int]),
    "e2e_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    "e2e_server_destroy": (C.c_int, [C.c_void_p]),
}

_lib = None
_lock = threading.Lock()


def lib():
    """Load libe2edp.so (fails loudly if it was not built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"{LIB_PATH} is missing: build it with `make -C e2e_gpu_dp_b200/csrc` "
                    "(there is no CPU fallback)")
            L = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            _lib = L
    return _lib


def check(status: int) -> None:
    if status != E2E_OK:
        msg = lib().e2e_last_error()
        raise E2EError(status, msg.decode() if msg else "")
