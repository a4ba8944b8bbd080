"""The environment generator's CPU restatement against the reference's own output.

tests/golden/env_*.npz were written by the reference's
build_environment_DG_with_westward_clouds (tests/golden/make_env_golden.py);
the oracle must reproduce every array bit for bit (same numpy / scipy calls,
the reference's Python float expressions).
"""
import os

import numpy as np
import pytest

from oracle import envgen as OE

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden(name):
    return np.load(os.path.join(HERE, "golden", f"{name}.npz"))


@pytest.mark.parametrize("name", ["env_a", "env_b"])
def test_oracle_matches_reference_generator(name):
    z = _golden(name)
    cfg = OE.config_from_golden(z)
    out = OE.generate(**cfg)
    assert np.array_equal(out["R_vel"], z["R_vel"]) and np.array_equal(out["R_phi"], z["R_phi"])
    for k in OE.FILES:
        assert out[k].dtype == z[k].dtype and out[k].shape == z[k].shape, k
        assert np.array_equal(out[k], z[k]), (k, float(np.max(np.abs(out[k] - z[k]))))
    n = cfg["n_modes"]
    assert np.allclose(out["svals_vel"], z["svals_vel"], rtol=1e-12, atol=1e-12 * z["svals_vel"].max())
    assert out["svals_vel"].shape[1] >= n


def test_oracle_mean_is_a_sequential_sum():
    # the GPU generator sums the samples in order; numpy's mean over axis 1 does too
    z = _golden("env_a")
    R = z["R_vel"]
    s = R[:, 0, :].copy()
    for k in range(1, R.shape[1]):
        s = s + R[:, k, :]
    assert np.array_equal(R.mean(axis=1), s / R.shape[1])


def test_oracle_cloud_and_obstacles_on_reference_grid():
    z = _golden("env_c")
    cfg = OE.config_from_golden(z)
    G = cfg["init_gsize"] * cfg["interpolate_degree"]
    stride = int(z["grid_stride"])
    s = OE.cloud(G, cfg["nt"], cfg["dxy"] / cfg["interpolate_degree"], cfg["A_sc"])
    assert np.array_equal(s[..., ::stride, ::stride], z["all_s_mat"])
    m = OE.obstacles(G, cfg["nt"], cfg["dyn_obstacle_data"])
    assert np.array_equal(m[..., ::stride, ::stride], z["obstacle_mask"])


def test_interp_table_equals_griddata():
    from scipy.interpolate import griddata

    from e2e_gpu_dp_b200.envgen import grid_ticks, interp_table
    rng = np.random.default_rng(3)
    for g, dxy, d in [(6, 2 / 6, 2), (4, 0.5, 1), (25, 2 / 25, 8), (7, 0.3, 3)]:
        vert, wgt = interp_table(g, dxy, d)
        xs = grid_ticks(g, dxy)
        xg, yg = np.meshgrid(xs, np.flip(xs))
        pts = np.stack([xg.flatten(), yg.flatten()], 1)
        nx = grid_ticks(g * d, dxy / d)
        nxg, nyg = np.meshgrid(nx, np.flip(nx))
        vals = rng.standard_normal(g * g).astype(np.float32)
        ref = griddata(pts, vals, (nxg, nyg), method="linear").astype(np.float32)
        v64 = vals.astype(np.float64)
        o = np.zeros(len(vert))
        for j in range(3):  # griddata's order: out = 0; out += c_j v_j
            o = o + wgt[:, j] * v64[np.maximum(vert[:, j], 0)]
        o[vert[:, 0] < 0] = np.nan
        assert np.array_equal(np.isnan(o.reshape(nxg.shape)), np.isnan(ref))
        assert np.array_equal(np.nan_to_num(o.astype(np.float32).reshape(nxg.shape)), np.nan_to_num(ref))
