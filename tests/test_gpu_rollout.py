"""GPU policy rollout (e2e_rollout) against the oracle and the reference's trajectories.

The kernel uses the oracle's fma-chain velocity and the reference's float32
scalar arithmetic otherwise, so outcomes, travel times, final cells and
energies must equal the oracle's bit for bit, and (through the pinned oracle)
the reference's trajectories stored in tests/golden/rollout_*.npz.
"""
import os

import numpy as np
import pytest

from e2e_gpu_dp_b200 import api
from oracle import rollout as RO
from tests.helpers import golden, problem

pytestmark = pytest.mark.gpu

NAMES = ["t_time", "t_custom", "c1"]


@pytest.mark.parametrize("name", NAMES)
def test_rollout_equals_oracle_and_reference(name):
    prob, fields = problem(name)
    pol = golden(name)["policy"].astype(np.int64)
    fx = np.load(os.path.join(os.path.dirname(__file__), "golden", f"rollout_{name}.npz"))
    for k, st in enumerate(fx["starts"]):
        r = api.rollout(prob, fields, pol.astype(np.int32), st)
        o = RO.rollout(prob, fields, pol, st, dot="fma")
        for key in ("success", "travel_time", "final_tij", "energy_cons", "energy_col", "net_energy"):
            assert np.array_equal(r[key], o[key]), (name, k, key)
        assert np.array_equal(r["success"], fx[f"success_{k}"])
        m = RO.metrics(o)
        s = r["stats"]
        assert s["n"] == prob.nrzns and s["success_rate"] == m["success_rate"]
        assert abs(s["mean_time"] - m["mean_travel_time"]) < 1e-9


def test_rollout_from_device_policy_after_gpu_solve():
    torch = pytest.importorskip("torch")
    prob, fields = problem("c1")
    m = api.build_model(prob, fields)
    V, pi, _ = m.solve(method="layered")
    m.free()
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in fields.items()}
    r = api.rollout(prob, dev, torch.from_numpy(pi).cuda(), (25, 47), n_rzns=200)
    o = RO.rollout(prob, fields, pi.astype(np.int64), (25, 47), n_rzns=200, dot="fma")
    assert np.array_equal(r["success"], o["success"]) and np.array_equal(r["final_tij"], o["final_tij"])


def test_rollout_reports_states_without_an_action():
    prob, fields = problem("t_time")
    pol = golden("t_time")["policy"].astype(np.int64).astype(np.int32)
    pol[8 * prob.gsize + 12] = -1  # the start cell at t = 0
    r = api.rollout(prob, fields, pol, (8, 12))
    assert np.all(r["success"] == -2) and r["stats"]["invalid"] == prob.nrzns
