"""GPU parity of the fused build+backup pass (e2e_build_solve).

It backs every layer up as soon as it is built, so it never stores the model;
its values and policy must equal, bit for bit, those of building the model and
running the layered solve (which the other GPU tests tie to the Jacobi solve,
the FP64 oracle and the reference).
"""
import numpy as np
import pytest

from e2e_gpu_dp_b200 import api
from e2e_gpu_dp_b200._lib import E2EError
from tests.helpers import PARITY, problem

pytestmark = pytest.mark.gpu

NAMES = PARITY + ["c1"]


@pytest.fixture(scope="module")
def solved():
    cache = {}

    def get(name):
        if name not in cache:
            prob, fields = problem(name)
            m = api.build_model(prob, fields)
            V, pi, st = m.solve(method="layered")
            cache[name] = (prob, fields, m.info(), V, pi, st)
            m.free()
        return cache[name]

    return get


@pytest.mark.parametrize("name", NAMES)
def test_fused_equals_build_then_layered_solve(solved, name):
    prob, fields, info, V, pi, _ = solved(name)
    Vf, pif, st = api.build_solve(prob, fields)
    assert np.array_equal(Vf, V), float(np.max(np.abs(Vf - V)))
    assert np.array_equal(pif, pi)
    assert st["n_rows"] == info["n_rows"]
    assert st["nnz"] == info["nnz"]
    assert st["dropped"] == info["dropped"] and st["overflow_rows"] == info["overflow_units"]
    assert st["launches"] >= 1  # one cooperative launch per pass (a pass re-runs for a larger pool)


def test_fused_dense_rows_are_backed_up(solved):
    prob, fields, info, V, pi, _ = solved("t_wide")
    assert info["overflow_units"] > 0  # rows that left the 8x8 window use dense histograms
    Vf, pif, st = api.build_solve(prob, fields)
    assert st["overflow_rows"] > 0
    assert np.array_equal(Vf, V) and np.array_equal(pif, pi)


def test_fused_device_fields_and_outputs(solved):
    torch = pytest.importorskip("torch")
    prob, fields, info, V, pi, _ = solved("t_custom")
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in fields.items()}
    Vd = torch.full((prob.ns,), float("nan"), dtype=torch.float32, device="cuda")
    pid = torch.full((prob.ns,), -7, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    _, _, st = api.build_solve(prob, dev, value=Vd, policy=pid, stream=s)
    torch.cuda.synchronize()
    assert st["h2d_bytes"] == 0
    assert np.array_equal(Vd.cpu().numpy(), V) and np.array_equal(pid.cpu().numpy(), pi)


def test_fused_repeatable(solved):
    prob, fields, info, V, pi, _ = solved("c1")
    for _ in range(2):
        Vf, pif, _ = api.build_solve(prob, fields)
        assert np.array_equal(Vf, V) and np.array_equal(pif, pi)


def test_fused_rejects_bad_arguments(solved):
    torch = pytest.importorskip("torch")
    prob, fields, *_ = solved("t_time")
    with pytest.raises(ValueError):
        api.build_solve(prob, fields, value=torch.empty(prob.ns, device="cuda"))
    # a null field pointer through the C ABI: an error status, nothing launched
    import ctypes as C
    from e2e_gpu_dp_b200 import _lib
    where, f, keep = api._fields_ptrs(fields)
    f.mask = None
    cp = api.c_problem(prob)
    st = _lib.FusedStats()
    V = np.zeros(prob.ns, np.float32)
    rc = _lib.lib().e2e_build_solve(C.byref(cp), C.byref(f), where, None, V.ctypes.data, _lib.E2E_HOST,
                                    C.byref(st), None)
    assert rc == _lib.E2E_ERR_INVALID
    with pytest.raises(E2EError):
        _lib.check(rc)
