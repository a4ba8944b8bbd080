"""The property behind the builder's in-window chunks, on the reference's own
arithmetic (the oracle reproduces the reference's next cells bit for bit).

A plain builder warp skips its per-sample window test for a chunk of
realisations when the landing bins of two corners of the chunk's velocity
bounding box, (vx min, vy max) and (vx max, vy min), lie in the row's window.
That is exact because the reference's landing cell is monotone in each
velocity component: non-decreasing in vx for the column, non-increasing in vy
for the row, every step of move() (advection, clamps, snapping) rounding a
monotone function.  Here the velocity of realisation r is made exactly Y[r]
(mean flow 0, one mode of 1), the Y are sorted and packed around every cell
edge a sample can reach, and every action of every cell must then land on
columns (rows) that never step back.
"""
import dataclasses

import numpy as np

from e2e_gpu_dp_b200.problem import config
from oracle import pyoracle as O


def _edge_hugging_values(prob, rng, n_uniform=1500):
    """Sorted float32 velocities: uniform ones plus, for every cell centre and
    heading, the velocities that put the landing within a few ulps of a cell
    edge (the snapping coordinate's .5 boundaries)."""
    speed, angle = prob.actions()
    cs, sn = O.host_trig(angle)
    xs, _ = prob.grid_ticks()
    vals = [rng.uniform(-2.5, 2.5, n_uniform).astype(np.float32)]
    edges = np.arange(0, prob.gsize + 1, dtype=np.float64)  # x = k: the column changes
    for x1 in xs[::3].astype(np.float64):
        for F, c, s in zip(speed.astype(np.float64), cs.astype(np.float64), sn.astype(np.float64)):
            for off in (c, s):
                t = (edges - x1 - F * off) / prob.dt
                t = t[np.abs(t) < 2.5].astype(np.float32)
                vals.append(t)
                vals.append(np.nextafter(t, np.float32(np.inf)))
                vals.append(np.nextafter(t, np.float32(-np.inf)))
    v = np.unique(np.concatenate(vals).astype(np.float32))
    return np.sort(v)


def _fields(prob, Y, axis):
    g, nt = prob.gsize, prob.nt
    zeros = np.zeros((nt, g, g), np.float32)
    ones = np.ones((nt, 1, g, g), np.float32)
    f = {"u": zeros.copy(), "v": zeros.copy(),
         "ui": ones.copy() if axis == "x" else np.zeros_like(ones),
         "vi": ones.copy() if axis == "y" else np.zeros_like(ones),
         "Yi": np.ascontiguousarray(np.broadcast_to(Y[None, :, None], (nt, len(Y), 1))).astype(np.float32),
         "s": zeros.copy(), "mask": np.zeros((nt, g, g), np.int32)}
    return f


def test_landing_cell_is_monotone_in_each_velocity_component():
    base, _ = config("t_custom")  # 16 headings, unit spacing
    rng = np.random.default_rng(7)
    probe = dataclasses.replace(base, nt=3, nmodes=1, nrzns=8)
    Y = _edge_hugging_values(probe, rng)
    prob = dataclasses.replace(probe, nrzns=len(Y))
    checked = changes = 0
    for axis in ("x", "y"):
        fields = _fields(prob, Y, axis)
        for cell in range(prob.ncells):
            for a in range(prob.num_actions):
                i2, j2, _, _ = O.samples(prob, fields, 0, cell, a)
                if axis == "x":
                    assert np.all(np.diff(j2) >= 0), (cell, a)
                    assert np.all(i2 == i2[0]), (cell, a)
                    changes += int(np.count_nonzero(np.diff(j2)))
                else:
                    assert np.all(np.diff(i2) <= 0), (cell, a)
                    assert np.all(j2 == j2[0]), (cell, a)
                    changes += int(np.count_nonzero(np.diff(i2)))
                checked += 1
    assert checked == 2 * prob.ncells * prob.num_actions
    # the samples do cross cell edges: several steps per (cell, action) on average
    assert changes > 3 * checked
