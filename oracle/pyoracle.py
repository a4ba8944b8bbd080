"""ctypes front end of the CPU oracle (oracle/e2e_oracle.c).

ORACLE -- test infrastructure only: imported by tests/, by
``__graft_entry__.smoke()`` and by the cpu-baseline leg of ``bench.py`` as the
checker; never by the product package.

Builds ``oracle/_build/liboracle.so`` with ``make -C oracle`` on first use.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading
from typing import Dict, Optional, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None
_lock = threading.Lock()


class _Problem(C.Structure):
    _fields_ = [
        ("gsize", C.c_int32), ("nt", C.c_int32), ("nrzns", C.c_int32), ("nmodes", C.c_int32),
        ("num_actions", C.c_int32), ("reward_type", C.c_int32), ("i_term", C.c_int32),
        ("j_term", C.c_int32), ("term_subgrid_size", C.c_int32), ("neighb_gsize", C.c_int32),
        ("dt", C.c_float), ("r_outbound", C.c_float), ("r_terminal", C.c_float),
        ("alpha", C.c_float),
    ]


class _Fields(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_float)) for n in ("u", "v", "ui", "vi", "Yi", "s")] + [
        ("mask", C.POINTER(C.c_int32))
    ]


class _Rows(C.Structure):
    _fields_ = [
        ("n_rows", C.c_int64), ("nnz", C.c_int64),
        ("row_ptr", C.POINTER(C.c_int64)), ("col", C.POINTER(C.c_int64)),
        ("cnt", C.POINTER(C.c_uint32)), ("R", C.POINTER(C.c_float)),
        ("dropped", C.c_uint64), ("misbinned", C.c_uint64), ("near_edge", C.c_uint64),
    ]


def build() -> str:
    """Compile the oracle library (idempotent)."""
    src = os.path.join(_HERE, "e2e_oracle.c")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build()
            L = C.CDLL(_LIB_PATH)
            fp = C.POINTER(C.c_float)
            L.orc_build_rows.argtypes = [C.POINTER(_Problem), C.POINTER(_Fields), fp, fp, fp, fp, fp,
                                         C.c_int64, C.c_int64, C.c_int, C.POINTER(_Rows)]
            L.orc_build_rows.restype = C.c_int
            L.orc_rows_free.argtypes = [C.POINTER(_Rows)]
            L.orc_samples.argtypes = [C.POINTER(_Problem), C.POINTER(_Fields), fp, fp, fp, fp, fp,
                                      C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int32),
                                      C.POINTER(C.c_int32), fp, C.POINTER(C.c_int32)]
            L.orc_action_trig.argtypes = [fp, C.c_int, fp, fp]
            vp = C.c_void_p
            L.orc_vi_f64.argtypes = [C.c_int64, C.c_int, C.c_int64, vp, vp, vp, vp, C.c_double, vp,
                                     C.c_int, C.c_double, C.c_int, vp, vp, vp]
            L.orc_vi_f64.restype = C.c_int
            L.orc_vi_f32.argtypes = [C.c_int64, C.c_int, C.c_int64, vp, vp, vp, vp, C.c_int32, vp,
                                     C.c_float, C.c_int, vp, vp, vp]
            L.orc_vi_f32.restype = C.c_int
            L.orc_vi_f64_layers.argtypes = [C.c_int64, C.c_int, C.c_int, vp, vp, vp, vp, C.c_double, vp,
                                            vp, C.c_int, vp, vp, vp]
            L.orc_vi_f64_layers.restype = C.c_int
            _lib = L
    return _lib


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _prob_struct(prob) -> _Problem:
    return _Problem(prob.gsize, prob.nt, prob.nrzns, prob.nmodes, prob.num_actions,
                    prob.reward_type, prob.i_term, prob.j_term, prob.term_subgrid_size,
                    prob.neighb_gsize, prob.dt, prob.r_outbound, prob.r_terminal, prob.alpha)


def _fields_struct(fields: Dict[str, np.ndarray], keep: list) -> _Fields:
    arrs = {}
    for k in ("u", "v", "ui", "vi", "Yi", "s"):
        a = np.ascontiguousarray(fields[k], dtype=np.float32)
        keep.append(a)
        arrs[k] = _fp(a)
    m = np.ascontiguousarray(fields["mask"], dtype=np.int32)
    keep.append(m)
    return _Fields(arrs["u"], arrs["v"], arrs["ui"], arrs["vi"], arrs["Yi"], arrs["s"],
                   m.ctypes.data_as(C.POINTER(C.c_int32)))


def host_trig(angles: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    a = np.ascontiguousarray(angles, dtype=np.float32)
    c = np.empty_like(a)
    s = np.empty_like(a)
    lib().orc_action_trig(_fp(a), len(a), _fp(c), _fp(s))
    return c, s


def build_rows(prob, fields, trig: Optional[Tuple[np.ndarray, np.ndarray]] = None,
               r0: int = 0, r1: Optional[int] = None, nthreads: int = 1) -> Dict[str, np.ndarray]:
    """Rows [r0, r1) of the state-major transition model (row = s*Na + a)."""
    L = lib()
    n_rows_total = (prob.nt - 1) * prob.ncells * prob.num_actions
    if r1 is None:
        r1 = n_rows_total
    keep: list = []
    P = _prob_struct(prob)
    Fs = _fields_struct(fields, keep)
    xs, ys = prob.grid_ticks()
    speed, angle = prob.actions()
    if trig is None:
        trig = host_trig(angle)
    cosv = np.ascontiguousarray(trig[0], dtype=np.float32)
    sinv = np.ascontiguousarray(trig[1], dtype=np.float32)
    out = _Rows()
    rc = L.orc_build_rows(C.byref(P), C.byref(Fs), _fp(xs), _fp(ys), _fp(speed), _fp(cosv),
                          _fp(sinv), r0, r1, nthreads, C.byref(out))
    if rc != 0:
        L.orc_rows_free(C.byref(out))
        raise RuntimeError(f"orc_build_rows failed ({rc})")
    n, nnz = out.n_rows, out.nnz
    res = {
        "row_ptr": np.ctypeslib.as_array(out.row_ptr, shape=(n + 1,)).copy(),
        "col": np.ctypeslib.as_array(out.col, shape=(max(nnz, 1),))[:nnz].copy(),
        "cnt": np.ctypeslib.as_array(out.cnt, shape=(max(nnz, 1),))[:nnz].copy(),
        "R": np.ctypeslib.as_array(out.R, shape=(max(n, 1),))[:n].copy(),
        "dropped": int(out.dropped), "misbinned": int(out.misbinned),
        "near_edge": int(out.near_edge),
    }
    L.orc_rows_free(C.byref(out))
    return res


def build_model(prob, fields, trig=None, nthreads: int = 4) -> Dict[str, np.ndarray]:
    """Whole state-major model: CSR over rows of layers 0..nt-2 plus the full
    R (Ns*Na, last layer zero as in src/build_model.cu:1173-1176)."""
    rows = build_rows(prob, fields, trig=trig, nthreads=nthreads)
    Na = prob.num_actions
    R = np.zeros(prob.ns * Na, dtype=np.float32)
    R[: len(rows["R"])] = rows["R"]
    rows["R_full"] = R
    return rows


def samples(prob, fields, T: int, cell: int, a: int, trig=None):
    """Per-realisation next cell, reward and near-edge flag of one (t, cell, a)."""
    L = lib()
    keep: list = []
    P = _prob_struct(prob)
    Fs = _fields_struct(fields, keep)
    xs, ys = prob.grid_ticks()
    speed, angle = prob.actions()
    if trig is None:
        trig = host_trig(angle)
    cosv = np.ascontiguousarray(trig[0], dtype=np.float32)
    sinv = np.ascontiguousarray(trig[1], dtype=np.float32)
    n = prob.nrzns
    i2 = np.empty(n, np.int32)
    j2 = np.empty(n, np.int32)
    r = np.empty(n, np.float32)
    ne = np.empty(n, np.int32)
    ip = C.POINTER(C.c_int32)
    L.orc_samples(C.byref(P), C.byref(Fs), _fp(xs), _fp(ys), _fp(speed), _fp(cosv), _fp(sinv),
                  T, cell, a, i2.ctypes.data_as(ip), j2.ctypes.data_as(ip), _fp(r),
                  ne.ctypes.data_as(ip))
    return i2, j2, r, ne


def vi_f64(Ns: int, Na: int, n_row_states: int, row_ptr, col, cnt=None, val=None, scale=1.0,
           R=None, mode: int = 1, thresh: float = 1e-12, max_iter: int = 100000):
    """FP64 value iteration (mode 1 = backward sweep, mode 0 = Jacobi)."""
    L = lib()
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
    col = np.ascontiguousarray(col, dtype=np.int64)
    cnt_a = None if cnt is None else np.ascontiguousarray(cnt, dtype=np.uint32)
    val_a = None if val is None else np.ascontiguousarray(val, dtype=np.float32)
    R = np.ascontiguousarray(R, dtype=np.float32)
    V = np.zeros(Ns, np.float64)
    pi = np.zeros(Ns, np.int32)
    res = np.zeros(1, np.float64)
    it = L.orc_vi_f64(Ns, Na, n_row_states, row_ptr.ctypes.data, col.ctypes.data,
                      None if cnt_a is None else cnt_a.ctypes.data,
                      None if val_a is None else val_a.ctypes.data, float(scale), R.ctypes.data,
                      mode, thresh, max_iter, V.ctypes.data, pi.ctypes.data, res.ctypes.data)
    return V, pi, it, float(res[0])


def vi_f32(Ns: int, Na: int, n_row_states: int, row_ptr, col, cnt=None, val=None, nrzns=1,
           R=None, thresh: float = 0.1, max_iter: int = 100000):
    """FP32 Jacobi value iteration with the reference's float semantics."""
    L = lib()
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
    col = np.ascontiguousarray(col, dtype=np.int64)
    cnt_a = None if cnt is None else np.ascontiguousarray(cnt, dtype=np.uint32)
    val_a = None if val is None else np.ascontiguousarray(val, dtype=np.float32)
    R = np.ascontiguousarray(R, dtype=np.float32)
    V = np.zeros(Ns, np.float32)
    pi = np.zeros(Ns, np.int32)
    res = np.zeros(1, np.float32)
    it = L.orc_vi_f32(Ns, Na, n_row_states, row_ptr.ctypes.data, col.ctypes.data,
                      None if cnt_a is None else cnt_a.ctypes.data,
                      None if val_a is None else val_a.ctypes.data, int(nrzns), R.ctypes.data,
                      float(thresh), max_iter, V.ctypes.data, pi.ctypes.data, res.ctypes.data)
    return V, pi, it, float(res[0])


def to_reference_coo(prob, model: Dict[str, np.ndarray]):
    """Reference on-disk layout (save_master_Coos_to_file, src/build_model.cu:1246-1314):
    action-major concatenation; within an action, time-major then cell, S2 ascending;
    S1 = a*Ns + t*ncells + cell; val = count/nrzns in float; R laid out [a][s]."""
    Na, Ns = prob.num_actions, prob.ns
    rp = model["row_ptr"]
    n_rows = len(rp) - 1
    lens = np.diff(rp)
    row_ids = np.arange(n_rows, dtype=np.int64)
    a_of_row = row_ids % Na
    s_of_row = row_ids // Na
    order_rows = np.lexsort((s_of_row, a_of_row))           # by a, then s
    starts = rp[:-1][order_rows]
    ln = lens[order_rows]
    idx = np.concatenate([np.arange(st, st + l) for st, l in zip(starts, ln)]) if len(ln) else np.zeros(0, np.int64)
    S1 = np.repeat(a_of_row[order_rows] * Ns + s_of_row[order_rows], ln).astype(np.int64)
    S2 = model["col"][idx].astype(np.int64)
    val = (model["cnt"][idx].astype(np.float32) / np.float32(prob.nrzns)).astype(np.float32)
    R_sa = model["R_full"].reshape(Ns, Na)
    R_ref = np.ascontiguousarray(R_sa.T).reshape(-1)
    return S1, S2, val, R_ref


def vi_f64_layers(ncells: int, nt: int, Na: int, row_ptr, col, cnt, scale: float, R, policy=None,
                  nthreads: int = 1):
    """FP64 backward induction over a time-layered state-major CSR with int32
    next states and uint16/uint32 counts (the library's layout, e.g. as copied
    down from the device), the states of a layer on ``nthreads`` threads.
    Returns (V64, pi64, gap): gap[s] = best Q - Q(s, policy[s]) in FP64 when a
    policy is given, else None."""
    L = lib()
    Ns = ncells * nt
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
    col = np.ascontiguousarray(col, dtype=np.int32)
    cnt = np.asarray(cnt)
    if cnt.dtype == np.uint16:
        c16, c32 = np.ascontiguousarray(cnt), None
    else:
        c16, c32 = None, np.ascontiguousarray(cnt, dtype=np.uint32)
    R = np.ascontiguousarray(R, dtype=np.float32)
    if len(R) != Ns * Na:
        raise ValueError("R needs ns * Na entries")
    pol = None if policy is None else np.ascontiguousarray(policy, dtype=np.int32)
    V = np.empty(Ns, np.float64)
    pi = np.empty(Ns, np.int32)
    gap = None if pol is None else np.empty(Ns, np.float64)
    rc = L.orc_vi_f64_layers(ncells, nt, Na, row_ptr.ctypes.data, col.ctypes.data,
                             None if c32 is None else c32.ctypes.data,
                             None if c16 is None else c16.ctypes.data, float(scale), R.ctypes.data,
                             None if pol is None else pol.ctypes.data, int(nthreads), V.ctypes.data,
                             pi.ctypes.data, None if gap is None else gap.ctypes.data)
    if rc != 0:
        raise RuntimeError("orc_vi_f64_layers failed")
    return V, pi, gap
