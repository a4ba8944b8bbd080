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
              stream=None, schedule: int = 0) -> Tuple:
        """Value iteration.  ``method``: "layered" (backward sweep + verification
        sweep) or "jacobi" (reference semantics).  With ``value``/``policy`` CUDA
        tensors the results stay on the device; otherwise numpy arrays are returned.
        ``schedule``: the ``schedule`` word of e2e_vi_opts (0 = automatic; bits 0-3
        warps per chunk, bit 8 set: bits 4-7 sweep tuning)."""
        inf = self.info()
        ns = inf["ns"]
        o = _lib.ViOpts(1 if method == "layered" else 0, threshold, max_iter, timeout_s,
                        1 if fp64_check else 0, schedule)
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


def solve_batch(models, values, policies, schedule: int = 0, stream=None) -> Dict:
    """Layered solves of many models in one persistent launch (e2e_spvi_solve_batch).
    ``values`` / ``policies``: CUDA tensors (float32 / int32), one per model, of
    its ``ns`` states.  Returns the batch statistics."""
    n = len(models)
    hs = (C.c_void_p * n)(*[m.handle for m in models])
    vs = (C.c_void_p * n)(*[v.data_ptr() for v in values])
    ps = (C.c_void_p * n)(*[p.data_ptr() for p in policies])
    o = _lib.ViOpts(1, 0.1, 0, 0.0, 0, schedule)
    st = _lib.BatchStats()
    check(lib().e2e_spvi_solve_batch(hs, n, C.byref(o), vs, ps, C.byref(st), _stream_ptr(stream)))
    return {f: getattr(st, f) for f, _ in _lib.BatchStats._fields_}


def build_models(probs, fields_list, count_type: str = "auto", workers: int = 4):
    """Many builds at once (e2e_build_models): ``workers`` host threads, one
    stream each.  Fields all on the host or all CUDA tensors."""
    n = len(probs)
    keep = []
    fs = (_lib.Fields * n)()
    where = None
    for i, fl in enumerate(fields_list):
        w, f, k = _fields_ptrs(fl)
        if where is None:
            where = w
        elif w != where:
            raise ValueError("fields must all be on the host or all on the device")
        fs[i] = f
        keep.append(k)
    ps = (_lib.Problem * n)(*[c_problem(p) for p in probs])
    o = _lib.BuildOpts(_COUNT[count_type], 0, 0, 0, 0)
    out = (C.c_void_p * n)()
    check(lib().e2e_build_models(ps, fs, n, where if where is not None else _lib.E2E_HOST, C.byref(o),
                                 workers, out))
    del keep
    return [Model(out[i], probs[i]) for i in range(n)]


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


def _fields_ptrs(fields: Dict):
    """(where, Fields struct, keep-alive list) for host numpy or CUDA tensor fields."""
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
    return where, f, keep


class Server:
    """The request server of the C ABI (e2e_server_*): resident fields, cached
    base models, continuous batching of plan requests on one GPU."""

    def __init__(self, hbm_budget: int = 0, max_batch: int = 0, schedule: int = 0):
        o = _lib.ServerOpts(hbm_budget, max_batch, schedule)
        h = C.c_void_p()
        check(lib().e2e_server_create(C.byref(o), C.byref(h)))
        self._h = h

    def add_field(self, prob: Problem, fields: Dict) -> int:
        where, f, keep = _fields_ptrs(fields)
        cp = c_problem(prob)
        fid = C.c_int32()
        check(lib().e2e_server_add_field(self._h, C.byref(cp), C.byref(f), where, C.byref(fid)))
        del keep
        return fid.value

    def submit(self, field_id: int, headings: int, target, start, keep_outputs: bool = False,
               tag: int = 0) -> int:
        r = _lib.Request(field_id, headings, int(target[0]), int(target[1]), int(start[0]), int(start[1]),
                         1 if keep_outputs else 0, 0, tag)
        rid = C.c_int64()
        check(lib().e2e_server_submit(self._h, C.byref(r), C.byref(rid)))
        return rid.value

    def cancel(self, request_id: int) -> None:
        """Cancel a queued request (e2e_server_cancel); its result comes back
        from poll() with status E2E_ERR_CANCELLED."""
        check(lib().e2e_server_cancel(self._h, request_id))

    def poll(self, max_results: int = 1024, wait_s: float = 0.0):
        buf = (_lib.Result * max_results)()
        n = C.c_int32()
        check(lib().e2e_server_poll(self._h, buf, max_results, C.byref(n), wait_s))
        return [{f: getattr(buf[i], f) for f, _ in _lib.Result._fields_} for i in range(n.value)]

    def fetch(self, request_id: int, ns: int):
        V = np.empty(ns, np.float32)
        pi = np.empty(ns, np.int32)
        check(lib().e2e_server_fetch(self._h, request_id, V.ctypes.data, pi.ctypes.data, _lib.E2E_HOST))
        return V, pi

    def stats(self) -> Dict:
        st = _lib.ServerStats()
        check(lib().e2e_server_get_stats(self._h, C.byref(st)))
        return {f: getattr(st, f) for f, _ in _lib.ServerStats._fields_}

    def close(self) -> None:
        if self._h:
            lib().e2e_server_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build_solve(prob: Problem, fields: Dict, value=None, policy=None, stream=None):
    """Build and solve in one backward pass without storing the model
    (e2e_build_solve): layer t's rows are backed up as soon as they are built.
    ``value`` / ``policy``: optional CUDA tensors of ns float32 / int32 to fill;
    otherwise host numpy arrays are returned.  Returns (V, policy, stats)."""
    where, f, keep = _fields_ptrs(fields)
    st = _lib.FusedStats()
    cp = c_problem(prob)
    if value is not None or policy is not None:
        if value is None or policy is None or not (_is_device(value) and _is_device(policy)):
            raise ValueError("pass both value and policy as CUDA tensors, or neither")
        if value.numel() != prob.ns or policy.numel() != prob.ns:
            raise ValueError("value and policy need ns entries")
        V, pi = value, policy
        out_where, vptr, pptr = _lib.E2E_DEVICE, value.data_ptr(), policy.data_ptr()
    else:
        V = np.empty(prob.ns, np.float32)
        pi = np.empty(prob.ns, np.int32)
        out_where, vptr, pptr = _lib.E2E_HOST, V.ctypes.data, pi.ctypes.data
    check(lib().e2e_build_solve(C.byref(cp), C.byref(f), where, pptr, vptr, out_where, C.byref(st),
                                _stream_ptr(stream)))
    del keep
    return V, pi, {k: getattr(st, k) for k, _ in _lib.FusedStats._fields_}


def rollout(prob: Problem, fields: Dict, policy, start, n_rzns: int = 0, stream=None,
            interpolate: bool = False) -> Dict:
    """Follow ``policy`` (ns int32, numpy or CUDA tensor) from ``start`` (i, j)
    for each realisation (e2e_rollout).  ``interpolate``: actions after the
    first interpolated from the four cells around the position (the reference
    script's with_policy_interp).  Returns per-realisation arrays and the
    summary of the reference's get_metrics."""
    where, f, keep = _fields_ptrs(fields)
    n = n_rzns if n_rzns > 0 else prob.nrzns
    if _is_device(policy):
        pw, pptr = _lib.E2E_DEVICE, policy.data_ptr()
    else:
        pol = np.ascontiguousarray(policy, dtype=np.int32)
        keep.append(pol)
        pw, pptr = _lib.E2E_HOST, pol.ctypes.data
    succ = np.empty(n, np.int8)
    tt = np.empty(n, np.int32)
    en = np.empty((n, 3), np.float32)
    fin = np.empty((n, 3), np.int32)
    o = _lib.RolloutOpts(int(start[0]), int(start[1]), n, _lib.E2E_ROLLOUT_INTERP if interpolate else 0)
    st = _lib.RolloutStats()
    cp = c_problem(prob)
    check(lib().e2e_rollout(C.byref(cp), C.byref(f), where, pptr, pw, C.byref(o), succ.ctypes.data,
                            tt.ctypes.data, en.ctypes.data, fin.ctypes.data, C.byref(st), _stream_ptr(stream)))
    del keep
    out = {"success": succ, "travel_time": tt, "energy_cons": en[:, 0].astype(np.float64),
           "energy_col": en[:, 1].astype(np.float64), "net_energy": en[:, 2].astype(np.float64),
           "final_tij": fin}
    out["stats"] = {k: getattr(st, k) for k, _ in _lib.RolloutStats._fields_}
    return out
