"""The solve entry point that allocates no device memory.

Some callers of this library cannot call cudaMalloc: a serving loop whose
device memory is fully reserved by its own pool, or code running while another
framework's allocator owns the device.  e2e_spvi_solve_noalloc serves them: it
takes caller-provided device outputs and keeps its scratch in a fixed
file-scope device array.  These tests call it through the C ABI and compare it
with the regular e2e_spvi_solve, on two calls in a row (the array keeps the
previous call's contents, so the second call must not depend on them), check
that those calls leave the device's free memory unchanged, and solve a model
without time layers with the default options (Jacobi until the reference's
threshold, no limit on the number of sweeps).
"""
import ctypes as C
import os

import numpy as np
import pytest

from e2e_gpu_dp_b200 import _lib, api
from tests.helpers import VALUE_RTOL, problem, values_close

pytestmark = pytest.mark.gpu

MAX_STATES = ((32 << 20) - 256) // 4


def _buffers(ns):
    import torch

    V = torch.full((ns,), float("nan"), dtype=torch.float32, device="cuda")
    pi = torch.full((ns,), -7, dtype=torch.int32, device="cuda")
    return V, pi


def _noalloc(model, method, threshold=0.1, bufs=None, opts=True):
    import torch

    ns = model.info()["ns"]
    V, pi = bufs if bufs is not None else _buffers(ns)
    V.fill_(float("nan"))
    pi.fill_(-7)
    o = _lib.ViOpts(method, threshold, 0, 0.0, 0, 0)
    stats = _lib.ViStats()
    torch.cuda.synchronize()
    st = _lib.lib().e2e_spvi_solve_noalloc(model.handle, C.byref(o) if opts else None, pi.data_ptr(),
                                            V.data_ptr(), C.byref(stats), None)
    _lib.check(st)
    torch.cuda.synchronize()
    return V.cpu().numpy(), pi.cpu().numpy(), stats


@pytest.mark.parametrize("name", ["c1", "t_custom"])
@pytest.mark.parametrize("method", [1, 0])
def test_noalloc_matches_regular_solve_on_two_calls(name, method):
    prob, fields = problem(name)
    model = api.build_model(prob, fields)
    V_ref, pi_ref, st_ref = model.solve(method="layered" if method == 1 else "jacobi", threshold=0.1)
    for _ in range(2):
        V, pi, st = _noalloc(model, method)
        rel, _ = values_close(V, V_ref.astype(np.float64))
        assert rel <= VALUE_RTOL
        assert np.array_equal(pi, pi_ref)
        assert st.iterations == st_ref["iterations"]
        assert st.residual == st_ref["residual"]
    model.free()


def test_noalloc_leaves_free_device_memory_unchanged():
    """After a first call (module loading, the array's address), trimming the
    library's pool and cache, two more calls change nothing in the device's
    free memory: a call that went through the library's pool would have
    reserved memory that stays reserved until the next trim."""
    import torch

    prob, fields = problem("c1")
    model = api.build_model(prob, fields)
    bufs = _buffers(prob.ns)
    _noalloc(model, 1, bufs=bufs)
    _noalloc(model, 0, bufs=bufs)
    _lib.check(_lib.lib().e2e_memory_trim())
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for method in (1, 0):
        _noalloc(model, method, bufs=bufs)
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    model.free()


def _banded_model_dir(d, ncells=20, nt=6, nu=2, na=4):
    from tests.test_oracle_golden import banded_mdp

    Ns, na, S1, S2, val, R = banded_mdp(ncells, nt, nu, na)
    np.save(os.path.join(d, "master_cooS1.npy"), S1.astype(np.int32).reshape(-1, 1))
    np.save(os.path.join(d, "master_cooS2.npy"), S2.astype(np.int32).reshape(-1, 1))
    np.save(os.path.join(d, "master_cooVal.npy"), val.reshape(-1, 1))
    np.save(os.path.join(d, "master_R.npy"), R.reshape(-1, 1))
    np.save(os.path.join(d, "DP_relv_params.npy"), np.array([[Ns], [na]], np.int64))


def test_noalloc_model_without_layers_default_options(tmp_path):
    """A model read without prob_params has no time layers: the default is
    Jacobi with the regular solve's default sweep limit, like e2e_spvi_solve."""
    _banded_model_dir(str(tmp_path))
    model = api.Model.read_npy(str(tmp_path))
    inf = model.info()
    assert inf["count_type"] == 2
    V_ref, pi_ref, st_ref = model.solve(method="jacobi", threshold=0.1)
    for _ in range(2):
        V, pi, st = _noalloc(model, 0, opts=False)
        rel, _ = values_close(V, V_ref.astype(np.float64))
        assert rel <= VALUE_RTOL
        assert np.array_equal(pi, pi_ref)
        assert st.iterations == st_ref["iterations"] and st.residual < 0.1
    model.free()


def test_noalloc_rejects_models_above_its_capacity(tmp_path):
    ns = MAX_STATES + 1
    d = str(tmp_path)
    np.save(os.path.join(d, "master_cooS1.npy"), np.array([[0]], np.int32))
    np.save(os.path.join(d, "master_cooS2.npy"), np.array([[1]], np.int32))
    np.save(os.path.join(d, "master_cooVal.npy"), np.array([[1.0]], np.float32))
    np.save(os.path.join(d, "master_R.npy"), np.zeros((ns, 1), np.float32))
    np.save(os.path.join(d, "DP_relv_params.npy"), np.array([[ns], [1]], np.int64))
    model = api.Model.read_npy(d)
    with pytest.raises(_lib.E2EError) as ei:
        _noalloc(model, 0)
    assert ei.value.status == 7 and "at most" in str(ei.value)
    model.free()
