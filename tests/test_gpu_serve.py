"""The request server (e2e_server_*) against the plain per-request path.

The plain path builds the model with the request's target and heading set on
the field's own arrays and solves it (e2e_build_model + e2e_spvi_solve).  The
server re-targets a cached base model instead.  With the "time" reward (integer
dt, r_outbound, r_terminal) every reward sum is exact, so the results must be
bit-identical; a result must also be the same whether its request was solved
alone or in a batch with others.
"""
import numpy as np
import pytest

from e2e_gpu_dp_b200 import api
from e2e_gpu_dp_b200.workloads import with_target
from tests.helpers import VALUE_RTOL, problem, values_close

pytestmark = pytest.mark.gpu

INTEGER_FIELDS = ["t_time", "t_wide", "c1"]


def _plain(prob, fields, headings, target):
    p = with_target(prob, headings, target)
    m = api.build_model(p, fields)
    V, pi, _ = m.solve(method="layered")
    m.free()
    return V, pi


def _wait(srv, ids, timeout=60.0):
    got = {}
    import time
    t0 = time.time()
    while len(got) < len(ids) and time.time() - t0 < timeout:
        for r in srv.poll(wait_s=0.5):
            got[r["request_id"]] = r
    assert len(got) == len(ids)
    return got


@pytest.fixture(scope="module")
def server():
    srv = api.Server()
    fids = {}
    for name in INTEGER_FIELDS + ["t_custom"]:
        prob, fields = problem(name)
        fids[name] = (srv.add_field(prob, fields), prob, fields)
    yield srv, fids
    srv.close()


def test_served_equals_plain_build_and_solve(server):
    srv, fids = server
    rng = np.random.default_rng(3)
    cases = []
    for name in INTEGER_FIELDS:
        fid, prob, fields = fids[name]
        g = prob.gsize
        for headings in (prob.num_ac_angles, 16):
            tgt = (int(rng.integers(g)), int(rng.integers(g)))
            start = (int(rng.integers(g)), int(rng.integers(g)))
            rid = srv.submit(fid, headings, tgt, start, keep_outputs=True)
            cases.append((rid, name, prob, fields, headings, tgt, start))
    res = _wait(srv, [c[0] for c in cases])
    for rid, name, prob, fields, headings, tgt, start in cases:
        r = res[rid]
        assert r["status"] == 0, (name, r)
        ns = prob.ns
        V, pi = srv.fetch(rid, ns)
        Vp, pip = _plain(prob, fields, headings, tgt)
        assert np.array_equal(V, Vp), (name, headings, tgt)
        assert np.array_equal(pi, pip), (name, headings, tgt)
        s0 = start[0] * prob.gsize + start[1]
        assert r["value_at_start"] == V[s0] and r["action_at_start"] == pi[s0]


def test_non_integer_rewards_within_tolerance(server):
    srv, fids = server
    fid, prob, fields = fids["t_custom"]
    tgt, start = (5, 9), (1, 1)
    rid = srv.submit(fid, prob.num_ac_angles, tgt, start, keep_outputs=True)
    r = _wait(srv, [rid])[rid]
    assert r["status"] == 0
    V, pi = srv.fetch(rid, prob.ns)
    Vp, _ = _plain(prob, fields, prob.num_ac_angles, tgt)
    rel, _ = values_close(V, Vp.astype(np.float64))
    assert rel <= VALUE_RTOL


def test_same_result_alone_and_in_a_mix(server):
    srv, fids = server
    fid, prob, fields = fids["c1"]
    tgt, start = (30, 12), (3, 40)
    rid = srv.submit(fid, 8, tgt, start, keep_outputs=True)
    _wait(srv, [rid])
    V1, pi1 = srv.fetch(rid, prob.ns)
    rng = np.random.default_rng(11)
    ids = []
    for k in range(40):
        name = INTEGER_FIELDS[k % len(INTEGER_FIELDS)]
        f2, p2, _ = fids[name]
        g = p2.gsize
        ids.append(srv.submit(f2, int(rng.choice([8, 16])), (int(rng.integers(g)), int(rng.integers(g))),
                              (0, 0)))
        if k == 20:
            rid2 = srv.submit(fid, 8, tgt, start, keep_outputs=True)
            ids.append(rid2)
    res = _wait(srv, ids)
    assert all(r["status"] == 0 for r in res.values())
    assert res[rid2]["batch_size"] > 1
    V2, pi2 = srv.fetch(rid2, prob.ns)
    assert np.array_equal(V1, V2) and np.array_equal(pi1, pi2)


def _all_models_bytes(pa, fa, pb, fb):
    with api.Server() as srv:
        ia, ib = srv.add_field(pa, fa), srv.add_field(pb, fb)
        ids = [srv.submit(f, h, (1, 1), (0, 0)) for f in (ia, ib) for h in (8, 16)]
        _wait(srv, ids)
        return srv.stats()["bytes_in_use"]


def test_small_budget_evicts_and_stays_correct():
    prob_a, fields_a = problem("t_time")
    prob_b, fields_b = problem("t_wide")
    budget = int(0.75 * _all_models_bytes(prob_a, fields_a, prob_b, fields_b))
    with api.Server(hbm_budget=budget, max_batch=4) as srv:
        fa = srv.add_field(prob_a, fields_a)
        fb = srv.add_field(prob_b, fields_b)
        ids = []
        for k in range(6):
            f, p = (fa, prob_a) if k % 2 == 0 else (fb, prob_b)
            ids.append((srv.submit(f, 8 if k < 4 else 16, (k, k + 1), (1, 2), keep_outputs=True), f, p, k))
        res = _wait(srv, [i[0] for i in ids])
        st = srv.stats()
        assert st["models_evicted"] > 0 and st["failed"] == 0
        for rid, f, p, k in ids:
            fields = fields_a if f == fa else fields_b
            V, pi = srv.fetch(rid, p.ns)
            Vp, pip = _plain(p, fields, 8 if k < 4 else 16, (k, k + 1))
            assert np.array_equal(V, Vp) and np.array_equal(pi, pip)
            assert res[rid]["status"] == 0


def test_budget_below_any_model_fails_the_request():
    prob, fields = problem("t_time")
    with api.Server(hbm_budget=1 << 20) as srv:
        fid = srv.add_field(prob, fields)
        rid = srv.submit(fid, 8, (1, 1), (2, 2))
        r = _wait(srv, [rid])[rid]
        assert r["status"] != 0
        with pytest.raises(Exception):
            srv.submit(fid, 8, (prob.gsize, 0), (0, 0))  # target outside the grid
