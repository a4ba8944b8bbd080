"""Shared checks for the parity tests."""
from __future__ import annotations

import os

import numpy as np

from e2e_gpu_dp_b200.problem import config, make_fields

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# FP32 values against the FP64 oracle, normwise: max|V32 - V64| / max|V64|.
VALUE_RTOL = 1e-5
# Actions whose FP64 Q lies within this normwise band of the best are ties.
TIE_RTOL = 2e-5

# Small problems of the parity tests.  t_m10 / t_m8 carry the per-row shape of
# the 200x200x120 and 300x300x150 workloads (16 headings, 10 / 8 modes, 5000 /
# 2000 realisations), t_m6 6 modes and 32 actions; the energy problems cover
# the reward types 1-3 and custom1 the mixed one.
PARITY = ["t_time", "t_custom", "t_energy2", "t_wide", "t_m10", "t_m8", "t_m6", "t_energy1",
          "t_energy3", "t_half"]
# Problems whose rewards are integers: every reward sum is exact in float, so
# R is compared bit for bit (t_half's time step is 0.5: sums of halves and
# hundreds, exact too).
INTEGER_REWARDS = {"t_time", "t_wide", "c1", "t_m10", "t_m8", "t_m6", "t_half"}


def problem(name, seed=1234):
    prob, spec = config(name, seed)
    return prob, make_fields(prob, spec)


def golden(name):
    path = os.path.join(GOLDEN, f"ref_{name}.npz")
    return np.load(path)


def q_values_f64(prob, row_ptr, col, cnt, R_full, V64, n_row_states=None, val=None):
    """FP64 Q(s, a) = R + sum cnt/nrzns * V[col] for every state-major row."""
    Na = prob.num_actions
    Ns = prob.ns
    if n_row_states is None:
        n_row_states = (prob.nt - 1) * prob.ncells
    Q = R_full.astype(np.float64).reshape(Ns, Na).copy()
    rp = np.asarray(row_ptr, dtype=np.int64)
    n_rows = len(rp) - 1
    w = (np.asarray(cnt, np.float64) / prob.nrzns) if val is None else np.asarray(val, np.float64)
    contrib = w * V64[np.asarray(col, np.int64)]
    sums = np.zeros(n_rows)
    lens = np.diff(rp)
    nz = lens > 0
    if len(contrib):
        sums[nz] = np.add.reduceat(contrib, rp[:-1][nz])
    Q.reshape(-1)[:n_rows] += sums
    return Q


def policy_ok(Q64, pi, V64):
    """Every chosen action is within the tie band of the FP64 best action."""
    best = Q64.max(axis=1)
    band = TIE_RTOL * max(1.0, float(np.max(np.abs(V64))))
    chosen = Q64[np.arange(len(pi)), np.asarray(pi, np.int64)]
    bad = np.nonzero(chosen < best - band)[0]
    return bad


def values_close(V, V64):
    err = float(np.max(np.abs(np.asarray(V, np.float64) - V64)))
    scale = float(np.max(np.abs(V64)))
    return err / max(scale, 1e-30), err
