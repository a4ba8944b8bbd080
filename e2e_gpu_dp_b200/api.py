"""Python front end of the C ABI: build a transition model, solve it, and read
or write it in the reference's .npy layout.

Mirrors the reference's two-stage pipeline (src/Makefile:1-24):
``build_model`` (src/build_model.cu:926-1238) -> ``spvi_2`` (src/spvi_2.cu:730-796),
as function calls on device-resident data.  Fields may be numpy arrays (host,
copied in by the library) or CUDA tensors (device pointers, used in place).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Tuple

import numpy as np

from . import _lib
from ._lib import check, lib
from .problem import Problem

_COUNT = {"auto": _lib.E2E_COUNT_AUTO, "u16": _lib.E2E_COUNT_U16, "u32": _lib.E2E_COUNT_U32}


def c_problem(p: Problem) -> _lib.Problem:
    x0 = np.float32(p.dx) / np.float32(2)
    y0 = np.float32(p.dy) / np.float32(2)
    return _lib.Problem(
        p.gsize, p.num_actions, p.nrzns, p.F, p.dt, p.r_outbound, p.r_terminal, p.nmodes,
        p.i_term, p.j_term, p.nt, p.is_stationary, p.term_subgrid_size, p.reward_type,
        p.num_ac_speeds, p.num_ac_angles, p.dx, p.dy, p.neighb_gsize, p.alpha, float(x0),
        float(y0))


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        return None
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream)
    return int(stream)


def action_table(p: Problem) -> Dict[str, np.ndarray]:
    """Speeds, headings and the device's cosf/sinf of every action."""
    na = p.num_actions
    out = {k: np.zeros(na, np.float32) for k in ("speed", "angle", "cos", "sin")}
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
    cp = c_problem(p)
    check(lib().e2e_action_table(C.byref(cp), fp(out["speed"]), fp(out["angle"]), fp(out["cos"]),
                                 fp(out["sin"])))
    return out


def _is_device(x) -> bool:
    return hasattr(x, "data_ptr") and getattr(x, "is_cuda", False)


class Model:
    """Device-resident transition model (state-major CSR + R)."""

    def __init__(self, handle: int, prob: Optional[Problem] = None):
        self._h = C.c_void_p(handle)
        self.prob = prob

    @property
    def handle(self) -> C.c_void_p:
        if not self._h:
            raise RuntimeError("model already freed")
        return self._h

    def info(self) -> Dict:
        inf = _lib.ModelInfo()
        check(lib().e2e_model_get_info(self.handle, C.byref(inf)))
        return {f: getattr(inf, f) for f, _ in _lib.ModelInfo._fields_}

    def to_host(self) -> Dict[str, np.ndarray]:
        inf = self.info()
        n_rows, nnz, ns, na = inf["n_rows"], inf["nnz"], inf["ns"], inf["num_actions"]
        rp = np.zeros(n_rows + 1, np.int64)
        col = np.zeros(max(nnz, 1), np.int32)
        cnt = np.zeros(max(nnz, 1), np.uint32)
        R = np.zeros(ns * na, np.float32)
        check(lib().e2e_model_copy_to_host(self.handle, rp.ctypes.data, col.ctypes.data,
                                           cnt.ctypes.data, R.ctypes.data, None))
        out = {"row_ptr": rp, "col": col[:nnz], "cnt": cnt[:nnz], "R": R}
        if inf["count_type"] == _lib.E2E_VALUE_F32:
            out["val"] = out["cnt"].view(np.float32)
        return out

    def write_npy(self, dirpath: str, index_bits: int = 64, prob: Optional[Problem] = None):
        p = prob or self.prob
        cp = C.byref(c_problem(p)) if p is not None else None
        check(lib().e2e_model_write_npy(self.handle, cp, dirpath.encode(), index_bits))

    @classmethod
    def read_npy(cls, dirpath: str, stream=None) -> "Model":
        h = C.c_void_p()
        check(lib().e2e_model_read_npy(dirpath.encode(), C.byref(h), _stream_ptr(stream)))
        return cls(h.value)

    def solve(self, method: str = "layered", threshold: float = 0.1, max_iter: int = 0,
              timeout_s: float = 0.0, fp64_check: bool = False, value=None, policy=None,
              stream=None) -> Tuple:
        """Value iteration.  ``method``: "layered" (backward sweep + verification
        sweep) or "jacobi" (reference semantics).  With ``value``/``policy`` CUDA
        tensors the results stay on the device; otherwise numpy arrays are returned."""
        inf = self.info()
        ns = inf["ns"]
        o = _lib.ViOpts(1 if method == "layered" else 0, threshold, max_iter, timeout_s,
                        1 if fp64_check else 0, 0)
        stats = _lib.ViStats()
        if value is not None and hasattr(value, "data_ptr"):
            where = _lib.E2E_DEVICE if _is_device(value) else _lib.E2E_HOST
            st = lib().e2e_spvi_solve(self.handle, C.byref(o), policy.data_ptr(), value.data_ptr(),
                                      where, C.byref(stats), _stream_ptr(stream))
            V, pi = value, policy
        else:
            V = np.zeros(ns, np.float32)
            pi = np.zeros(ns, np.int32)
            st = lib().e2e_spvi_solve(self.handle, C.byref(o), pi.ctypes.data, V.ctypes.data,
                                      _lib.E2E_HOST, C.byref(stats), _stream_ptr(stream))
        check(st)
        return V, pi, {f: getattr(stats, f) for f, _ in _lib.ViStats._fields_}

    def free(self) -> None:
        if self._h:
            lib().e2e_model_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def build_model(prob: Problem, fields: Dict, count_type: str = "auto", stream=None) -> Model:
    """Monte-Carlo transition build of every (t, cell, action) row on the GPU."""
    keep = []
    if all(_is_device(fields[k]) for k in ("u", "v", "Yi", "s", "mask")):
        where = _lib.E2E_DEVICE
        ptr = {k: fields[k].data_ptr() for k in fields}
    else:
        where = _lib.E2E_HOST
        ptr = {}
        for k in ("u", "v", "ui", "vi", "Yi", "s", "mask"):
            a = np.ascontiguousarray(fields[k], dtype=np.int32 if k == "mask" else np.float32)
            keep.append(a)
            ptr[k] = a.ctypes.data
    f = _lib.Fields(ptr["u"], ptr["v"], ptr["ui"], ptr["vi"], ptr["Yi"], ptr["s"], ptr["mask"])
    o = _lib.BuildOpts(_COUNT[count_type], 0, 0, 0, 0)
    h = C.c_void_p()
    cp = c_problem(prob)
    check(lib().e2e_build_model(C.byref(cp), C.byref(f), where, C.byref(o), C.byref(h),
                                _stream_ptr(stream)))
    return Model(h.value, prob)
