"""Failure paths on the GPU, in the forms that fault nothing.

* Bounded device waits: the persistent layered sweep waits on grid barriers,
  the batched sweep and the fused build+backup on per-layer completion
  counters; every wait gives up
  after a limit, sets an error word and lets the launch drain, and the host
  returns E2E_ERR_DEVICE.  The test hook E2E_TEST_UNREACHABLE_WAIT=1 raises
  every wait's target by one so that no wait can complete, with the limit cut
  to 50 ms (E2E_WAIT_LIMIT_MS); afterwards the same context must solve
  normally, bit for bit as before.
* The host wall-clock limit of value iteration (timeout_s, the limit the
  reference's solver declares, src/spvi_2.cu:650-726) -> E2E_ERR_TIMEOUT.
* A queued server request cancelled -> its result carries E2E_ERR_CANCELLED.
"""
import os
import time

import numpy as np
import pytest

from e2e_gpu_dp_b200 import api
from e2e_gpu_dp_b200._lib import E2EError
from tests.helpers import problem

pytestmark = pytest.mark.gpu

E2E_ERR_TIMEOUT, E2E_ERR_DEVICE, E2E_ERR_CANCELLED, E2E_ERR_BUSY = 5, 8, 9, 10


class _UnreachableWaits:
    def __enter__(self):
        os.environ["E2E_TEST_UNREACHABLE_WAIT"] = "1"
        os.environ["E2E_WAIT_LIMIT_MS"] = "50"
        return self

    def __exit__(self, *exc):
        os.environ.pop("E2E_TEST_UNREACHABLE_WAIT", None)
        os.environ.pop("E2E_WAIT_LIMIT_MS", None)


@pytest.fixture(scope="module")
def model():
    prob, fields = problem("t_custom")
    m = api.build_model(prob, fields)
    V, pi, _ = m.solve(method="layered")
    yield prob, m, V, pi
    m.free()


def test_layered_barrier_wait_runs_out(model):
    prob, m, V, pi = model
    t0 = time.time()
    with _UnreachableWaits():
        with pytest.raises(E2EError) as ei:
            m.solve(method="layered")
    assert ei.value.status == E2E_ERR_DEVICE
    assert time.time() - t0 < 30
    V2, pi2, st = m.solve(method="layered")  # the context is still usable
    assert st["residual"] == 0.0
    assert np.array_equal(V2, V) and np.array_equal(pi2, pi)


def test_batched_completion_wait_runs_out(model):
    import torch

    prob, m, V, pi = model
    Vd = torch.empty(prob.ns, dtype=torch.float32, device="cuda")
    pid = torch.empty(prob.ns, dtype=torch.int32, device="cuda")
    sch = 1 | (1 << 4) | 0x100 | 0x200  # fixed schedule, direct launch (no graph)
    with _UnreachableWaits():
        with pytest.raises(E2EError) as ei:
            api.solve_batch([m], [Vd], [pid], schedule=sch)
    assert ei.value.status == E2E_ERR_DEVICE
    api.solve_batch([m], [Vd], [pid], schedule=sch)
    torch.cuda.synchronize()
    assert np.array_equal(Vd.cpu().numpy(), V) and np.array_equal(pid.cpu().numpy(), pi)


def test_fused_layer_wait_runs_out(model):
    prob, m, V, pi = model
    _, fields = problem("t_custom")
    t0 = time.time()
    with _UnreachableWaits():
        with pytest.raises(E2EError) as ei:
            api.build_solve(prob, fields)
    assert ei.value.status == E2E_ERR_DEVICE
    assert time.time() - t0 < 30
    Vf, pif = api.build_solve(prob, fields)[:2]  # the context is still usable
    assert np.array_equal(Vf, V) and np.array_equal(pif, pi)


def test_jacobi_wall_clock_limit(model):
    prob, m, V, pi = model
    with pytest.raises(E2EError) as ei:
        m.solve(method="jacobi", threshold=1e-30, max_iter=10000, timeout_s=1e-9)
    assert ei.value.status == E2E_ERR_TIMEOUT
    V2, pi2, _ = m.solve(method="jacobi", threshold=1e-30, max_iter=prob.nt + 3)
    assert np.array_equal(V2, V) and np.array_equal(pi2, pi)


def test_server_cancel_of_queued_requests():
    """One request at a time (max_batch 1), a burst of 60, the last 30
    cancelled at once: every request gets exactly one result; a cancel that
    succeeded gives E2E_ERR_CANCELLED, one that came too late (E2E_ERR_BUSY)
    leaves a normal result."""
    prob, fields = problem("c1")
    with api.Server(max_batch=1) as srv:
        fid = srv.add_field(prob, fields)
        rng = np.random.default_rng(11)
        ids = []
        for _ in range(60):
            tgt = (int(rng.integers(prob.gsize)), int(rng.integers(prob.gsize)))
            ids.append(srv.submit(fid, 8, tgt, (1, 1)))
        outcome = {}
        for rid in ids[30:]:
            try:
                srv.cancel(rid)
                outcome[rid] = E2E_ERR_CANCELLED
            except E2EError as e:
                assert e.status == E2E_ERR_BUSY
                outcome[rid] = 0
        with pytest.raises(E2EError) as ei:
            srv.cancel(10**9)
        assert ei.value.status == 1
        got = {}
        t0 = time.time()
        while len(got) < len(ids) and time.time() - t0 < 120:
            for r in srv.poll(wait_s=0.5):
                assert r["request_id"] not in got
                got[r["request_id"]] = r
        assert len(got) == len(ids)
        for rid in ids[:30]:
            assert got[rid]["status"] == 0
        for rid in ids[30:]:
            assert got[rid]["status"] == outcome[rid]
        assert sum(1 for v in outcome.values() if v == E2E_ERR_CANCELLED) > 0
        st = srv.stats()
        assert st["pending"] == 0
