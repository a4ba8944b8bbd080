"""GPU policy rollout (e2e_rollout) against the oracle and the reference's trajectories.

The kernel uses the oracle's fma-chain velocity and the reference's float32
scalar arithmetic otherwise, so outcomes, travel times, final cells and
energies must equal the oracle's bit for bit, and (through the pinned oracle)
the reference's trajectories stored in tests/golden/rollout_*.npz.

With interpolated actions (the reference script's with_policy_interp) the
heading's atan2 / cosine and the speed's root come from the device's math
library where the reference uses the host libm and NumPy's scalar power, so
trajectories are compared per realisation: outcome and final cell must agree
for at least 99 % of the realisations (they agree for all in these cases),
travel times where they agree, and energies within 1e-3 relative (interpolated
speeds depend continuously on the position, so last-bit differences add up
along a trajectory).
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


@pytest.mark.parametrize("name", NAMES)
def test_interpolated_rollout_agrees_with_reference(name):
    prob, fields = problem(name)
    pol = golden(name)["policy"].astype(np.int64)
    fx = np.load(os.path.join(os.path.dirname(__file__), "golden", f"rollout_interp_{name}.npz"))
    for k, st in enumerate(fx["starts"]):
        r = api.rollout(prob, fields, pol.astype(np.int32), st, interpolate=True)
        same = (r["success"] == fx[f"success_{k}"]) & np.all(r["final_tij"] == fx[f"final_tij_{k}"], axis=1)
        assert same.mean() >= 0.99, (name, k, float(same.mean()))
        assert np.array_equal(r["travel_time"][same], fx[f"travel_time_{k}"][same])
        for e in ("energy_cons", "energy_col", "net_energy"):
            ref = fx[f"{e}_{k}"][same]
            # interpolated speeds vary continuously with the position, so last-bit
            # differences accumulate along a trajectory: 1e-3 relative (the CPU
            # restatement with the kernel's fma velocity already differs by 3e-4)
            assert np.allclose(r[e][same], ref, rtol=1e-3, atol=1e-3 * max(1.0, float(np.max(np.abs(ref))))), e
        plain = api.rollout(prob, fields, pol.astype(np.int32), st)
        assert plain["stats"]["n"] == r["stats"]["n"]


def test_interpolated_rollout_near_the_target_uses_the_triangle_form():
    # c1 from (25, 47): 60 of its interpolations happen in a cell diagonal to
    # the target, where the reference interpolates on a triangle in float64 and
    # its position becomes float64 (the kernel's double movement path)
    prob, fields = problem("c1")
    pol = golden("c1")["policy"].astype(np.int64)
    r = api.rollout(prob, fields, pol.astype(np.int32), (25, 47), interpolate=True)
    o = RO.rollout(prob, fields, pol, (25, 47), dot="fma", interp=True)
    assert np.mean(r["success"] == o["success"]) >= 0.99
    assert r["stats"]["success_rate"] == pytest.approx(RO.metrics(o)["success_rate"], abs=0.01)
