"""Batched layered solves (e2e_spvi_solve_batch) against one-at-a-time solves.

Every state's value in the batched launch is the same FMA chain as in the
single-model sweep, so values and policies must be bit-identical, whatever the
schedule, with or without the CUDA graph, and on graph replays.
"""
import numpy as np
import pytest

from e2e_gpu_dp_b200 import api
from e2e_gpu_dp_b200._lib import E2EError
from tests.helpers import PARITY, problem

pytestmark = pytest.mark.gpu

NAMES = PARITY + ["c1"]


@pytest.fixture(scope="module")
def models():
    torch = pytest.importorskip("torch")
    out = []
    for name in NAMES:
        prob, fields = problem(name)
        m = api.build_model(prob, fields)
        # reference: Jacobi from V = 0 (independent of any buffer's earlier contents)
        V, pi, _ = m.solve(method="jacobi", threshold=1e-30, max_iter=prob.nt + 3)
        out.append((name, prob, m, V, pi))
    # one model with uint32 counts: a second layout group in the same batch
    prob, fields = problem("t_time")
    m32 = api.build_model(prob, fields, count_type="u32")
    out.append(("t_time_u32", prob, m32, out[0][3], out[0][4]))
    yield out
    for _, _, m, _, _ in out:
        m.free()
    del torch


def _outputs(models):
    import torch
    vs = [torch.full((p.ns,), float("nan"), dtype=torch.float32, device="cuda") for _, p, _, _, _ in models]
    ps = [torch.full((p.ns,), -7, dtype=torch.int32, device="cuda") for _, p, _, _, _ in models]
    return vs, ps


def _check(models, vs, ps):
    for (name, _, _, V, pi), v, p in zip(models, vs, ps):
        assert np.array_equal(v.cpu().numpy(), V), name
        assert np.array_equal(p.cpu().numpy(), pi), name


def test_batch_equals_single_solves_autotuned_and_replayed(models):
    vs, ps = _outputs(models)
    st = api.solve_batch([m for _, _, m, _, _ in models], vs, ps)
    assert st["jobs"] == len(models) and st["launches"] == 2  # two layout groups
    _check(models, vs, ps)
    # second call of the same shape: no tuning, replayed graph, fresh outputs
    vs2, ps2 = _outputs(models)
    st2 = api.solve_batch([m for _, _, m, _, _ in models], vs2, ps2)
    assert st2["tune_ms"] == 0.0
    _check(models, vs2, ps2)


@pytest.mark.parametrize("graph", [True, False])
def test_every_batch_schedule(models, graph):
    ms = [m for _, _, m, _, _ in models]
    for groups in (1, 2, 4, 8):
        for tune in (0, 1, 2, 4, 5):
            vs, ps = _outputs(models)
            sch = groups | (tune << 4) | 0x100 | (0 if graph else 0x200)
            api.solve_batch(ms, vs, ps, schedule=sch)
            _check(models, vs, ps)


def test_rule_based_schedule(models):
    ms = [m for _, _, m, _, _ in models]
    for sch in (0x400, 0x400 | 0x200, 0x400 | 4):
        vs, ps = _outputs(models)
        api.solve_batch(ms, vs, ps, schedule=sch)
        _check(models, vs, ps)


def test_batch_of_one_and_order_independence(models):
    import torch
    name, prob, m, V, pi = models[2]
    v = torch.empty(prob.ns, dtype=torch.float32, device="cuda")
    p = torch.empty(prob.ns, dtype=torch.int32, device="cuda")
    api.solve_batch([m], [v], [p])
    assert np.array_equal(v.cpu().numpy(), V) and np.array_equal(p.cpu().numpy(), pi)
    rev = list(reversed(models))
    vs, ps = _outputs(rev)
    api.solve_batch([mm for _, _, mm, _, _ in rev], vs, ps)
    _check(rev, vs, ps)


def test_batch_rejects_bad_schedule(models):
    vs, ps = _outputs(models[:1])
    with pytest.raises(E2EError):
        api.solve_batch([models[0][2]], vs, ps, schedule=3 | 0x100)


def test_concurrent_builds_equal_single_builds(models):
    """e2e_build_models on several host threads and streams gives the same models."""
    probs, fields = [], []
    for name in ("t_time", "t_custom", "t_wide", "c1"):
        p, f = problem(name)
        probs.append(p)
        fields.append(f)
    built = api.build_models(probs, fields, workers=3)
    for p, f, m in zip(probs, fields, built):
        ref = api.build_model(p, f)
        a, b = m.to_host(), ref.to_host()
        for k in ("row_ptr", "col", "cnt", "R"):
            assert np.array_equal(a[k], b[k]), (p.prob_name, k)
        ref.free()
        m.free()
