"""GPU parity: the CUDA builder and solver against the oracle and the reference.

Counts and next states are integer work and must match bit for bit; values
are FP32 and must lie within VALUE_RTOL (normwise) of the FP64 oracle, with
policies equal up to ties (tests/helpers.py).
"""
import os
import tempfile

import numpy as np
import pytest

from e2e_gpu_dp_b200 import api
from e2e_gpu_dp_b200._lib import E2EError
from oracle import pyoracle as O
from tests.golden.make_golden import decode
from tests.golden.make_golden import NAMES as REF_NAMES
from tests.helpers import (INTEGER_REWARDS, PARITY, VALUE_RTOL, golden, policy_ok, problem, q_values_f64,
                           values_close)

pytestmark = pytest.mark.gpu

SMALL = PARITY
NTHREADS = max(1, min(16, os.cpu_count() or 1))


def _device_trig(prob):
    tab = api.action_table(prob)
    return tab["cos"], tab["sin"]


@pytest.fixture(scope="module")
def built():
    cache = {}

    def get(name):
        if name not in cache:
            prob, fields = problem(name)
            trig = _device_trig(prob)
            model = api.build_model(prob, fields)
            orc = O.build_model(prob, fields, trig=trig, nthreads=NTHREADS)
            cache[name] = (prob, fields, model, model.to_host(), orc)
        return cache[name]

    return get


@pytest.mark.parametrize("name", SMALL)
def test_transitions_bit_exact_vs_oracle(built, name):
    prob, fields, model, h, orc = built(name)
    info = model.info()
    assert info["dropped"] == orc["dropped"] == 0
    assert info["n_rows"] == (prob.nt - 1) * prob.ncells * prob.num_actions
    assert np.array_equal(h["row_ptr"], orc["row_ptr"])
    assert np.array_equal(h["col"], orc["col"])
    assert np.array_equal(h["cnt"], orc["cnt"])
    n = len(orc["R"])
    if name in INTEGER_REWARDS:
        assert np.array_equal(h["R"][:n], orc["R"])
    else:
        tol = prob.nrzns * 1.2e-7 * float(np.max(np.abs(orc["R"])))
        assert float(np.max(np.abs(h["R"][:n] - orc["R"]))) <= tol
    assert not np.any(h["R"][n:])  # last layer: zero reward, no rows


def test_wide_spread_uses_dense_rows(built):
    prob, fields, model, h, orc = built("t_wide")
    assert model.info()["overflow_units"] > 0
    assert np.array_equal(h["cnt"], orc["cnt"])


@pytest.mark.parametrize("name", REF_NAMES)
def test_model_files_equal_reference(name):
    """The reference's own output files, bit for bit (Val, S1, S2; R for integer rewards)."""
    prob, fields = problem(name)
    fx = golden(name)
    ref = decode(prob, fx)
    model = api.build_model(prob, fields)
    with tempfile.TemporaryDirectory() as d:
        model.write_npy(d, index_bits=64)
        S1 = np.load(os.path.join(d, "master_cooS1.npy"))
        S2 = np.load(os.path.join(d, "master_cooS2.npy"))
        val = np.load(os.path.join(d, "master_cooVal.npy"))
        R = np.load(os.path.join(d, "master_R.npy"))
        assert S1.dtype == np.int64 and S1.shape == (len(ref["S1"]), 1)
        assert np.array_equal(S1.ravel(), ref["S1"])
        assert np.array_equal(S2.ravel(), ref["S2"])
        assert np.array_equal(val.ravel(), ref["val"])
        assert np.array_equal(np.load(os.path.join(d, "prob_params.npy")).ravel(), ref["prob_params"])
        assert np.array_equal(np.load(os.path.join(d, "DP_relv_params.npy")).ravel(), ref["DP_relv_params"])
        if name in INTEGER_REWARDS:
            assert np.array_equal(R.ravel(), ref["R"])
        else:
            tol = prob.nrzns * 1.2e-7 * float(np.max(np.abs(ref["R"])))
            assert float(np.max(np.abs(R.ravel() - ref["R"]))) <= tol


@pytest.mark.parametrize("name", SMALL)
def test_solve_against_fp64_oracle(built, name):
    prob, fields, model, h, orc = built(name)
    nrs = (prob.nt - 1) * prob.ncells
    V64, _, _, _ = O.vi_f64(prob.ns, prob.num_actions, nrs, orc["row_ptr"], orc["col"],
                            cnt=orc["cnt"], scale=prob.nrzns, R=orc["R_full"], mode=1)
    Q = q_values_f64(prob, orc["row_ptr"], orc["col"], orc["cnt"], orc["R_full"], V64)
    Vl, pil, sl = model.solve(method="layered", fp64_check=True)
    Vj, pij, sj = model.solve(method="jacobi", threshold=1e-30, max_iter=prob.nt + 3)
    rel, _ = values_close(Vl, V64)
    assert rel <= VALUE_RTOL
    assert len(policy_ok(Q, pil, V64)) == 0
    assert sl["residual"] == 0.0 and sl["iterations"] == 2
    assert sl["fp64_max_rel_err"] <= VALUE_RTOL
    # the model is a layered DAG: Jacobi reaches the same values, bit for bit
    assert sj["residual"] == 0.0 and sj["iterations"] <= prob.nt + 1
    assert np.array_equal(Vl, Vj) and np.array_equal(pil, pij)


def test_jacobi_reference_threshold_stops_like_reference(built):
    prob, fields, model, h, orc = built("t_time")
    fx = golden("t_time")
    V, pi, st = model.solve(method="jacobi", threshold=0.1)
    assert st["iterations"] == prob.nt  # the reference's spvi_2 reported nt iterations
    rel, _ = values_close(V, fx["value"].astype(np.float64))
    assert rel <= VALUE_RTOL


def test_device_fields_and_outputs(built):
    torch = pytest.importorskip("torch")
    prob, fields, model, h, orc = built("t_custom")
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in fields.items()}
    m2 = api.build_model(prob, dev, stream=torch.cuda.current_stream())
    h2 = m2.to_host()
    for k in ("row_ptr", "col", "cnt", "R"):
        assert np.array_equal(h2[k], h[k])
    V = torch.empty(prob.ns, dtype=torch.float32, device="cuda")
    pi = torch.empty(prob.ns, dtype=torch.int32, device="cuda")
    m2.solve(method="layered", value=V, policy=pi, stream=torch.cuda.current_stream())
    torch.cuda.synchronize()
    Vh, pih, _ = model.solve(method="layered")
    assert np.array_equal(V.cpu().numpy(), Vh) and np.array_equal(pi.cpu().numpy(), pih)


@pytest.mark.parametrize("bits", [64, 32])
def test_npy_round_trip(built, bits):
    prob, fields, model, h, orc = built("t_energy2")
    with tempfile.TemporaryDirectory() as d:
        model.write_npy(d, index_bits=bits)
        m2 = api.Model.read_npy(d)
        inf = m2.info()
        assert inf["count_type"] == 0  # exact counts recognised from count/nrzns
        h2 = m2.to_host()
        n_rows = len(h["row_ptr"]) - 1
        assert np.array_equal(h2["row_ptr"][: n_rows + 1], h["row_ptr"])
        assert np.all(h2["row_ptr"][n_rows:] == h["row_ptr"][-1])  # empty last-layer rows
        assert np.array_equal(h2["col"], h["col"]) and np.array_equal(h2["cnt"], h["cnt"])
        assert np.array_equal(h2["R"], h["R"])
        V1, p1, _ = model.solve(method="layered")
        V2, p2, _ = m2.solve(method="layered")
        assert np.array_equal(V1, V2) and np.array_equal(p1, p2)


def test_read_reference_files_and_solve():
    """spvi_2 drop-in: the reference's converted (int32) files in, reference results out."""
    prob, _ = problem("t_custom")
    fx = golden("t_custom")
    ref = decode(prob, fx)
    with tempfile.TemporaryDirectory() as d:
        np.save(os.path.join(d, "master_cooS1.npy"), ref["S1"].astype(np.int32).reshape(-1, 1))
        np.save(os.path.join(d, "master_cooS2.npy"), ref["S2"].astype(np.int32).reshape(-1, 1))
        np.save(os.path.join(d, "master_cooVal.npy"), ref["val"].reshape(-1, 1))
        np.save(os.path.join(d, "master_R.npy"), ref["R"].reshape(-1, 1))
        np.save(os.path.join(d, "DP_relv_params.npy"), ref["DP_relv_params"].reshape(-1, 1))
        np.save(os.path.join(d, "prob_params.npy"), ref["prob_params"].reshape(-1, 1))
        m = api.Model.read_npy(d)
        V, pi, st = m.solve(method="jacobi", threshold=0.1)
    assert st["iterations"] == prob.nt
    rel, _ = values_close(V, ref["value"].astype(np.float64))
    assert rel <= VALUE_RTOL


def test_banded_known_answer_on_gpu():
    from tests.test_oracle_golden import banded_mdp

    ncells, nt, nu, na = 20, 6, 2, 4
    Ns, na, S1, S2, val, R = banded_mdp(ncells, nt, nu, na)
    with tempfile.TemporaryDirectory() as d:
        np.save(os.path.join(d, "master_cooS1.npy"), S1.astype(np.int32).reshape(-1, 1))
        np.save(os.path.join(d, "master_cooS2.npy"), S2.astype(np.int32).reshape(-1, 1))
        np.save(os.path.join(d, "master_cooVal.npy"), val.reshape(-1, 1))
        np.save(os.path.join(d, "master_R.npy"), R.reshape(-1, 1))
        np.save(os.path.join(d, "DP_relv_params.npy"), np.array([[Ns], [na]], np.int64))
        m = api.Model.read_npy(d)
        assert m.info()["count_type"] == 2  # float values (no prob_params)
        V, pi, st = m.solve(method="jacobi", threshold=1e-6, max_iter=50)
    best = R.reshape(na, Ns).T[:, -1].astype(np.float64)
    Vx = np.zeros(Ns)
    for t in range(nt - 1, -1, -1):
        cont = 0.0 if t == nt - 1 else np.mean(Vx[(t + 1) * ncells:(t + 1) * ncells + nu])
        Vx[t * ncells:(t + 1) * ncells] = best[t * ncells:(t + 1) * ncells] + cont
    assert np.allclose(V, Vx, rtol=1e-6)
    assert np.all(pi == na - 1)


def test_invalid_problems_are_rejected():
    prob, fields = problem("t_time")
    bad = type(prob)(**{**prob.__dict__, "neighb_gsize": 4})
    with pytest.raises(E2EError) as ei:
        api.build_model(bad, fields)
    assert ei.value.status == 1
    many = type(prob)(**{**prob.__dict__, "num_ac_angles": 40})
    with pytest.raises(E2EError) as ei:
        api.build_model(many, fields)
    assert ei.value.status == 7


@pytest.mark.parametrize("name", ["t_time", "t_custom"])
def test_every_sweep_schedule_gives_identical_results(built, name):
    """Sweep schedules (warps per chunk, prefetch, kernel variant) change only
    the work split; every state's value is the same FMA chain, so results are
    bit-identical to the default schedule."""
    torch = pytest.importorskip("torch")
    prob, fields, model, h, orc = built(name)
    # reference: Jacobi from V = 0 reads nothing the caller's buffers held
    Vd, pid, _ = model.solve(method="jacobi", threshold=1e-30, max_iter=prob.nt + 3)
    for groups in (0, 1, 2, 4, 8):
        for tune in range(8):
            # outputs start as NaN: the in-place layered sweep must never read them unwritten
            V = torch.full((prob.ns,), float("nan"), device="cuda")
            pi = torch.full((prob.ns,), -7, dtype=torch.int32, device="cuda")
            _, _, st = model.solve(method="layered", schedule=groups | (tune << 4) | 0x100, value=V, policy=pi)
            torch.cuda.synchronize()
            assert st["residual"] == 0.0
            assert np.array_equal(V.cpu().numpy(), Vd) and np.array_equal(pi.cpu().numpy(), pid), (groups, tune)
    for tune in range(16):  # bit 3 of the tuning: the TMA-staged Jacobi sweep
        V, pi, _ = model.solve(method="jacobi", threshold=1e-30, max_iter=prob.nt + 3,
                               schedule=(tune << 4) | 0x100)
        assert np.array_equal(V, Vd) and np.array_equal(pi, pid), tune
    with pytest.raises(E2EError):
        model.solve(method="layered", schedule=3)


def test_count_widths_and_layouts_agree(built):
    """uint32 counts take the separate offset/count layout; the values are the
    same as the packed uint16 layout's."""
    prob, fields, model, h, orc = built("t_time")
    m32 = api.build_model(prob, fields, count_type="u32")
    assert m32.info()["count_type"] != model.info()["count_type"]
    for method in ("layered", "jacobi"):
        V16, pi16, _ = model.solve(method=method, threshold=1e-30, max_iter=prob.nt + 3)
        V32, pi32, _ = m32.solve(method=method, threshold=1e-30, max_iter=prob.nt + 3)
        assert np.array_equal(V16, V32) and np.array_equal(pi16, pi32)
    m32.free()
