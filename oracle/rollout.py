"""CPU restatement of the reference's policy rollout (test infrastructure only).

Follows the trajectory loop of Post_processing/plot_e2eGPU_policy.py:433-474
(``plot_exact_trajectory_set_DP`` without policy interpolation) and the
movement of Post_processing/grid_world.py:160-271 (``Grid.move_exact``) with
the action set of grid_world.py:322-360 (``timeOpt_grid``) and the grid ticks of
Post_processing/utils/setup_grid.py (``Test_grid`` branch), in NumPy float32
scalar arithmetic (NumPy 2 rules: a Python number combined with a float32
scalar stays float32).  The velocity of a realisation at a cell is
``u + ui . Y``:

* ``dot="numpy"`` - ``np.matmul`` as the reference (its summation order is the
  BLAS library's); pinned bit for bit against tests/golden/rollout_*.npz, which
  were produced by the reference's own Grid class;
* ``dot="fma"`` - a sequential fused multiply-add chain over the modes, the
  order the GPU kernel uses (float32 fma emulated exactly through float64: the
  product of two float32 is exact in float64).

Per realisation: outcome (1 reached the target, 0 failed, -1 never decided),
travel time (steps), energy terms (sum F^2, sum of mean scalar field, their
difference) and the final (t, i, j).

``interp=True`` restates the script's ``with_policy_interp`` branch
(plot_e2eGPU_policy.py:483-486, get_interpolated_action :174-198,
interpolate_action_angles :111-171, bilinear / triangle interpolation
:37-108): after the first step the action is interpolated from the policy of
the four cells around the vehicle's position, in the same NumPy expressions
(float32 small matrix products, a float64 weight vector for the triangle case,
NumPy scalar powers); pinned against tests/golden/rollout_interp_*.npz, which
the reference's own functions produced.
"""
import math
from typing import Dict, Tuple

import numpy as np

F32 = np.float32


def action_table(prob) -> Tuple[np.ndarray, np.ndarray]:
    """Speeds (float32) and headings (Python floats) of timeOpt_grid
    (grid_world.py:322-360): speeds F or (i+1)*F/n, headings round(i*2pi/n, 14),
    speeds outer, headings inner (itertools.product)."""
    params = prob.prob_params()
    F, ns, na = params[3], int(params[14]), int(params[15])
    if ns == 1:
        speeds = [F]
    else:
        dF = F / ns
        speeds = [(i + 1) * dF for i in range(ns)]
    angles = [round(i * 2 * math.pi / na, 14) for i in range(na)]
    sp = np.array([s for s in speeds for _ in angles], np.float32)
    an = np.array([a for _ in speeds for a in angles], np.float64)
    return sp, an


def _fma32(a, b, c):
    return F32(float(a) * float(b) + float(c))


def _divmod32(a, b):
    """NumPy's float32 floor division and remainder (the published divmod
    algorithm: fmod, exact quotient correction, floor with the 0.5 guard)."""
    a, b = F32(a), F32(b)
    mod = F32(math.fmod(float(a), float(b)))
    div = F32(F32(a - mod) / b)
    if mod != 0:
        if (b < 0) != (mod < 0):
            mod = F32(mod + b)
            div = F32(div - F32(1.0))
    else:
        mod = F32(math.copysign(0.0, float(b)))
    if div != 0:
        fl = F32(math.floor(float(div)))
        if F32(div - fl) > F32(0.5):
            fl = F32(fl + F32(1.0))
    else:
        fl = F32(math.copysign(0.0, float(a) / float(b)))
    return fl, mod


def _bilinear(x, y, xt, yt, vals):
    v11, v12, v21, v22 = vals
    x1, x2 = xt
    y1, y2 = yt
    denom = 1 / ((x2 - x1) * (y2 - y1))
    xv = np.array([x2 - x, x - x1]).reshape((1, 2))
    vm = np.array([[v11, v12], [v21, v22]])
    yv = np.array([y2 - y, y - y1]).reshape((2, 1))
    return (denom * np.matmul(xv, np.matmul(vm, yv)))[0][0]


def _triangle(x, y, pts, vals):
    (x1, y1), (x2, y2), (x3, y3) = pts
    V = np.array(vals)
    W = np.zeros((3,))
    den = (y2 - y3) * (x1 - x3) + (x3 - x2) * (y1 - y3)
    W[0] = (y2 - y3) * (x - x3) + (x3 - x2) * (y - y3)
    W[1] = (y3 - y1) * (x - x3) + (x1 - x3) * (y - y3)
    W[0] = W[0] / den
    W[1] = W[1] / den
    W[2] = 1 - W[0] - W[1]
    return np.dot(V, W)


def interp_action(pol, speeds, angles, xs, ys, g, t, i, j, x, y, endpos):
    """(speed, heading) interpolated from the policy of the cell (t, i, j) that
    holds (x, y) and its three neighbours towards (x, y)."""
    sgn = lambda d: -1 if d < 0 else 1  # noqa: E731
    dy_, dx_ = sgn(y - ys[g - 1 - i]), sgn(x - xs[j])
    sup = [(t, i, j), (t, i - dy_, j), (t, i, j + dx_), (t, i - dy_, j + dx_)]
    term = [1 if (si, sj) == endpos else 0 for (_, si, sj) in sup]
    acts = [int(pol[sj + g * si + g * g * st]) for (st, si, sj) in sup]
    F = [speeds[a] for a in acts]
    th = [angles[a] for a in acts]
    cx = [xs[sj] for (_, _, sj) in sup]
    cy = [ys[g - 1 - si] for (_, si, _) in sup]
    vx = [F[k] * math.cos(th[k]) for k in range(4)]
    vy = [F[k] * math.sin(th[k]) for k in range(4)]
    method = "bilinear"
    if term == [0, 0, 0, 0]:
        pass
    elif term in ([0, 0, 1, 1], [0, 0, 1, 0]):
        vx[2], vx[3], vy[2], vy[3] = vx[0], vx[1], vy[0], vy[1]
    elif term in ([0, 1, 0, 1], [0, 1, 0, 0]):
        vx[1], vx[3], vy[1], vy[3] = vx[0], vx[2], vy[0], vy[2]
    elif term == [0, 0, 0, 1]:
        method = "triangle"
    else:
        raise ValueError(f"terminal pattern {term} cannot occur")
    x1, y1, x2, y2 = cx[0], cy[0], cx[3], cy[3]
    if method == "bilinear":
        ivx = _bilinear(x, y, (x1, x2), (y1, y2), vx)
        ivy = _bilinear(x, y, (x1, x2), (y1, y2), vy)
    else:
        pts = [(x1, y1), (x1, y2), (x2, y1)]
        ivx = _triangle(x, y, pts, [vx[0], vx[1], vx[2]])
        ivy = _triangle(x, y, pts, [vy[0], vy[1], vy[2]])
    ang = (math.atan2(ivy, ivx) + 2 * np.pi) % (2 * np.pi)
    return (ivx ** 2 + ivy ** 2) ** 0.5, ang


def rollout(prob, fields: Dict[str, np.ndarray], policy: np.ndarray, start, n_rzns=None, dot="fma",
            interp=False):
    params = prob.prob_params()
    g, nt = int(params[0]), int(params[10])
    dx, dy, dt = params[16], params[17], params[4]
    tsg, it, jt = int(params[12]), int(params[8]), int(params[9])
    xs = [(dx / 2) + (i * dx) for i in range(g)]
    ys = [(dy / 2) + (i * dy) for i in range(g)]
    dj, di = np.abs(xs[1] - xs[0]), np.abs(ys[1] - ys[0])
    speeds, angles = action_table(prob)
    u, v, ui, vi, Y, s_mat, mask = (fields[k] for k in ("u", "v", "ui", "vi", "Yi", "s", "mask"))
    nm = ui.shape[1]
    nrz = Y.shape[1] if n_rzns is None else n_rzns
    pol = np.asarray(policy).astype(np.int64)

    def term(i, j):
        return it <= i < it + tsg and jt <= j < jt + tsg

    def vel(t, i, j, rzn):
        if dot == "numpy":
            return (u[t, i, j] + np.matmul(ui[t, :, i, j], Y[t, rzn, :]),
                    v[t, i, j] + np.matmul(vi[t, :, i, j], Y[t, rzn, :]))
        ax = ay = F32(0)
        for k in range(nm):
            ax = _fma32(ui[t, k, i, j], Y[t, rzn, k], ax)
            ay = _fma32(vi[t, k, i, j], Y[t, rzn, k], ay)
        return F32(u[t, i, j] + ax), F32(v[t, i, j] + ay)

    out = {k: [] for k in ("success", "travel_time", "energy_cons", "energy_col", "net_energy", "final")}
    for rzn in range(nrz):
        t, i, j = 0, int(start[0]), int(start[1])
        x, y = xs[j], ys[g - 1 - i]
        a = int(pol[j + g * i + g * g * t])
        act = (speeds[a], angles[a])
        success = None
        e_cons = e_col = e_net = 0
        travel = 0
        for _ in range(nt):
            if success is None:
                vx, vy = vel(t, i, j, rzn)
                rad1 = s_mat[t, i, j]
                if not term(i, j) and t < nt - 1:          # move_exact (:162-269)
                    thrust, angle = act
                    vnx = (thrust * math.cos(angle)) + vx
                    vny = (thrust * math.sin(angle)) + vy
                    xn = x + (vnx * dt)
                    yn = y + (vny * dt)
                    if xn > xs[-1]:
                        xn = xs[-1]
                    elif xn < xs[0]:
                        xn = xs[0]
                    if yn > ys[-1]:
                        yn = ys[-1]
                    elif yn < ys[0]:
                        yn = ys[0]
                    x, y = xn, yn
                    xind, remx = _divmod32(xn - xs[0], dj)
                    yind, remy = _divmod32(-(yn - ys[-1]), di)
                    if remx >= 0.5 * dj:
                        xind = xind + 1
                    if remy >= 0.5 * di:
                        yind = yind + 1
                    if not (math.isnan(xind) or math.isnan(yind)):
                        i, j = int(yind), int(xind)
                    t += 1
                rad2 = s_mat[t, i, j]
                travel += 1
                e_cons += (1 * act[0]) ** 2
                e_col += (1 * (rad2 + rad1) / 2)
                e_net += (1 * (act[0] ** 2)) - (1 * (rad2 + rad1) / 2)
            if i == 0 or i == g - 1 or j == 0 or j == g - 1 or mask[t, i, j] == 1:
                success = False
            if (not term(i, j)) and t < nt - 1 and success is None:
                if interp:
                    act = interp_action(pol, speeds, angles, xs, ys, g, t, i, j, x, y, (it, jt))
                else:
                    a = int(pol[j + g * i + g * g * t])
                    act = (speeds[a], angles[a])
            elif term(i, j):
                success = True
            else:
                success = False
        out["success"].append(-1 if success is None else int(success))
        out["travel_time"].append(travel)
        out["energy_cons"].append(e_cons)
        out["energy_col"].append(e_col)
        out["net_energy"].append(e_net)
        out["final"].append((t, i, j))
    return {"success": np.array(out["success"], np.int8), "travel_time": np.array(out["travel_time"], np.int32),
            "energy_cons": np.array(out["energy_cons"], np.float64),
            "energy_col": np.array(out["energy_col"], np.float64),
            "net_energy": np.array(out["net_energy"], np.float64),
            "final_tij": np.array(out["final"], np.int32)}


def metrics(r) -> Dict[str, float]:
    """get_metrics (plot_e2eGPU_policy.py:776-797): success rate, and the means
    of travel time and energies over the successful realisations."""
    ok = r["success"] == 1
    n = len(r["success"])
    res = {"success_rate": float(ok.sum()) / n if n else 0.0}
    for k in ("travel_time", "energy_cons", "energy_col", "net_energy"):
        res[f"mean_{k}"] = float(np.mean(r[k][ok])) if ok.any() else 0.0
    return res
