"""The solve entry point that allocates no device memory.

Some callers of this library cannot call cudaMalloc: a serving loop whose
device memory is fully reserved by its own pool, or code running while another
framework's allocator owns the device.  e2e_spvi_solve_noalloc serves them: it
takes caller-provided device outputs and keeps its scratch in a fixed
file-scope device array.  These tests call it through the C ABI and compare it
with the regular e2e_spvi_solve, on two calls in a row (the array keeps the
previous call's contents, so the second call must not depend on them).
"""
import ctypes as C
import os

import numpy as np
import pytest

from e2e_gpu_dp_b200 import _lib, api
from tests.helpers import VALUE_RTOL, problem, values_close

pytestmark = pytest.mark.gpu

MAX_STATES = ((32 << 20) - 8192 * 8) // 4


def _noalloc(model, method, threshold=0.1):
    import torch

    ns = model.info()["ns"]
    V = torch.full((ns,), float("nan"), dtype=torch.float32, device="cuda")
    pi = torch.full((ns,), -7, dtype=torch.int32, device="cuda")
    o = _lib.ViOpts(method, threshold, 0, 0.0, 0, 0)
    stats = _lib.ViStats()
    torch.cuda.synchronize()
    st = _lib.lib().e2e_spvi_solve_noalloc(model.handle, C.byref(o), pi.data_ptr(), V.data_ptr(),
                                            C.byref(stats), None)
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
