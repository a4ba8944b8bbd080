"""The rollout oracle against the reference's own trajectories.

tests/golden/rollout_<name>.npz were produced by the reference's Grid class
(Post_processing/grid_world.py) following the reference's solved policies
(tests/golden/make_rollout_golden.py).  The oracle restatement must reproduce
them bit for bit with NumPy's dot product; with the GPU's fma-chain dot product
it may differ only where a velocity rounding moves a trajectory across a cell
edge, which these cases never do.
"""
import os

import numpy as np
import pytest

from oracle import rollout as RO
from tests.helpers import golden, problem

NAMES = ["t_time", "t_custom", "c1"]


def test_numpy_divmod_restatement():
    rng = np.random.default_rng(1)
    for _ in range(5000):
        a = np.float32(rng.uniform(-60, 60))
        b = np.float32(rng.choice([1.0, 0.5, 0.25, 1.5, 2.0, 3.0]))
        fl, md = RO._divmod32(a, b)
        assert fl == a // b and md == a % b


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("dot", ["numpy", "fma"])
def test_oracle_reproduces_reference_trajectories(name, dot):
    prob, fields = problem(name)
    pol = golden(name)["policy"].astype(np.int64)
    fx = np.load(os.path.join(os.path.dirname(__file__), "golden", f"rollout_{name}.npz"))
    for k, st in enumerate(fx["starts"]):
        r = RO.rollout(prob, fields, pol, st, dot=dot)
        assert np.array_equal(r["success"], fx[f"success_{k}"])
        assert np.array_equal(r["travel_time"], fx[f"travel_time_{k}"])
        assert np.array_equal(r["final_tij"], fx[f"final_tij_{k}"])
        for e in ("energy_cons", "energy_col", "net_energy"):
            assert np.array_equal(r[e], fx[f"{e}_{k}"])
    m = RO.metrics(r)
    assert 0.0 <= m["success_rate"] <= 1.0


@pytest.mark.parametrize("name", NAMES)
def test_oracle_interpolated_policy_reproduces_reference(name):
    # tests/golden/rollout_interp_<name>.npz: the reference's get_interpolated_action
    # (with_policy_interp) after the first step; the restatement uses the same
    # NumPy expressions, so with NumPy's dot product it agrees bit for bit
    prob, fields = problem(name)
    pol = golden(name)["policy"].astype(np.int64)
    fx = np.load(os.path.join(os.path.dirname(__file__), "golden", f"rollout_interp_{name}.npz"))
    for k, st in enumerate(fx["starts"]):
        r = RO.rollout(prob, fields, pol, st, dot="numpy", interp=True)
        for key in ("success", "travel_time", "final_tij", "energy_cons", "energy_col", "net_energy"):
            assert np.array_equal(r[key], fx[f"{key}_{k}"]), (name, k, key)
