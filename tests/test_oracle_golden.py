"""Pin the CPU oracle to the reference itself.

The fixtures in tests/golden/ are outputs of the reference's own programs
(src/build_model.cu -> convert -> src/spvi_2.cu, compiled unmodified for
sm_100a and run on a B200 on the seeded inputs of problem.config(name);
recipe in tests/golden/make_golden.py).  These tests run on the CPU.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as O
from tests.golden.make_golden import NAMES, decode, fields_digest
from tests.helpers import VALUE_RTOL, golden, policy_ok, problem, q_values_f64, values_close

from tests.helpers import INTEGER_REWARDS  # noqa: E402
NTHREADS = max(1, min(8, os.cpu_count() or 1))


def _oracle_model(name):
    prob, fields = problem(name)
    fx = golden(name)
    trig = None
    if "device_trig" in fx.files:
        trig = (fx["device_trig"][0], fx["device_trig"][1])
    m = O.build_model(prob, fields, trig=trig, nthreads=NTHREADS)
    return prob, fields, fx, m, trig is not None


@pytest.mark.parametrize("name", NAMES)
def test_inputs_regenerate_bit_for_bit(name):
    prob, fields = problem(name)
    fx = golden(name)
    assert fields_digest(fields) == bytes(fx["fields_sha256"]).hex()
    assert np.array_equal(fx["prob_params"], prob.prob_params())
    assert list(fx["DP_relv_params"]) == [prob.ns, prob.num_actions]


def _pair_counts(S1, S2, cnt):
    key = S1.astype(np.int64) * (1 << 32) + S2.astype(np.int64)
    return dict(zip(key.tolist(), cnt.tolist()))


@pytest.mark.parametrize("name", NAMES)
def test_oracle_transitions_match_reference(name):
    prob, fields, fx, m, exact_trig = _oracle_model(name)
    ref = decode(prob, fx)
    S1, S2, val, R = O.to_reference_coo(prob, m)
    cnt = np.repeat(np.diff(m["row_ptr"]), 1)  # noqa: F841 (shape check only)
    assert m["dropped"] == 0 and m["misbinned"] == 0
    if exact_trig or name != "c1":
        # identical next cells for every sample: identical COO, bit for bit
        assert np.array_equal(S1, ref["S1"])
        assert np.array_equal(S2, ref["S2"])
        assert np.array_equal(val, ref["val"])
    else:
        # host cosf may differ from the device's in the last bit; then only samples
        # within 1e-6 of a cell edge may land in the neighbouring cell
        a = _pair_counts(S1, S2, np.rint(val * prob.nrzns).astype(np.int64))
        b = _pair_counts(ref["S1"], ref["S2"], ref["count"])
        moved = sum(abs(a.get(k, 0) - b.get(k, 0)) for k in set(a) | set(b)) // 2
        assert moved <= m["near_edge"], (moved, m["near_edge"])
        assert moved <= 1e-6 * prob.nrzns * len(m["row_ptr"])
    Rref = ref["R"]
    if name in INTEGER_REWARDS and (exact_trig or name != "c1"):
        assert np.array_equal(R, Rref)
    else:
        # float rewards: the reference sums with float atomics in arbitrary order
        tol = prob.nrzns * 1.2e-7 * float(np.max(np.abs(Rref)))
        assert float(np.max(np.abs(R - Rref))) <= tol


@pytest.mark.parametrize("name", NAMES)
def test_reference_values_against_fp64_oracle(name):
    prob, fields, fx, m, _ = _oracle_model(name)
    ref = decode(prob, fx)
    nrs = (prob.nt - 1) * prob.ncells
    V64, pi64, _, _ = O.vi_f64(prob.ns, prob.num_actions, nrs, m["row_ptr"], m["col"],
                               cnt=m["cnt"], scale=prob.nrzns, R=m["R_full"], mode=1)
    rel, _ = values_close(ref["value"], V64)
    assert rel <= VALUE_RTOL
    Q = q_values_f64(prob, m["row_ptr"], m["col"], m["cnt"], m["R_full"], V64)
    assert len(policy_ok(Q, ref["policy"], V64)) == 0


@pytest.mark.parametrize("name", ["t_time", "t_custom"])
def test_jacobi_equals_backward_sweep(name):
    """The model is a time-layered DAG, so Jacobi from V=0 reaches the
    backward-induction values exactly (in FP64: bit for bit) after nt sweeps."""
    prob, fields = problem(name)
    m = O.build_model(prob, fields, nthreads=NTHREADS)
    nrs = (prob.nt - 1) * prob.ncells
    args = (prob.ns, prob.num_actions, nrs, m["row_ptr"], m["col"])
    Vb, pib, _, _ = O.vi_f64(*args, cnt=m["cnt"], scale=prob.nrzns, R=m["R_full"], mode=1)
    Vj, pij, it, res = O.vi_f64(*args, cnt=m["cnt"], scale=prob.nrzns, R=m["R_full"], mode=0,
                                thresh=1e-300, max_iter=prob.nt + 3)
    assert it <= prob.nt + 1 and res == 0.0
    assert np.array_equal(Vb, Vj) and np.array_equal(pib, pij)


def banded_mdp(ncells=20, nt=6, nu=2, na=4):
    """The synthetic MDP of the reference's (commented) get_mdp_model_test,
    src/spvi_2.cu:507-560: each row has nu entries of probability 1/nu into
    cells 0..nu-1 of the next layer; R[i] = 10*(i // Ns) + i over the
    action-major index i.  Returns the reference-layout COO."""
    Ns = ncells * nt
    nnz_per_ac = ncells * nu * (nt - 1)
    i = np.arange(nnz_per_ac * na, dtype=np.int64)
    rows = ((i % nnz_per_ac) // nu) + Ns * (i // nnz_per_ac)
    col_st = (((i % nnz_per_ac) // (ncells * nu)) + 1) * ncells
    cols = col_st + (i % nu)
    vals = np.full(len(i), 1.0 / nu, dtype=np.float32)
    R = np.array([10 * (k // Ns) + k for k in range(Ns * na)], dtype=np.float32)
    return Ns, na, rows, cols, vals, R


def coo_to_state_major(Ns, na, S1, S2, val):
    a = S1 // Ns
    s = S1 % Ns
    row = s * na + a
    order = np.argsort(row, kind="stable")
    counts = np.bincount(row, minlength=Ns * na)
    rp = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return rp, S2[order].astype(np.int64), val[order]


def test_banded_known_answer():
    ncells, nt, nu, na = 20, 6, 2, 4
    Ns, na, S1, S2, val, R = banded_mdp(ncells, nt, nu, na)
    rp, col, v = coo_to_state_major(Ns, na, S1, S2, val)
    Rsa = R.reshape(na, Ns).T.reshape(-1)
    V, pi, it, _ = O.vi_f64(Ns, na, Ns, rp, col, val=v, R=Rsa, mode=0, thresh=1e-12)
    # closed form: R grows with the action index, so the last action is best
    # everywhere; V(layer t, cell c) = R(na-1, s) + mean of V(layer t+1, cells 0..nu-1)
    Vx = np.zeros(Ns)
    best = Rsa.reshape(Ns, na)[:, -1].astype(np.float64)
    for t in range(nt - 1, -1, -1):
        sl = slice(t * ncells, (t + 1) * ncells)
        cont = 0.0 if t == nt - 1 else np.mean(Vx[(t + 1) * ncells:(t + 1) * ncells + nu])
        Vx[sl] = best[sl] + cont
    assert np.allclose(V, Vx, rtol=0, atol=1e-9)
    assert np.all(pi == na - 1)
    assert it == nt + 1 or it == nt
