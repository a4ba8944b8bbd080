"""Golden vectors of the reference's policy rollout (trajectory evaluation).

The reference evaluates a solved policy by following it from a start cell for
every realisation of the velocity field (Post_processing/plot_e2eGPU_policy.py:
376-474, ``plot_exact_trajectory_set_DP`` without policy interpolation),
moving with ``Grid.move_exact`` (Post_processing/grid_world.py:160-271), and
summarising success, travel time and energies (:776-797, ``get_metrics``).

This script runs that movement code itself: it imports ``timeOpt_grid`` /
``Grid`` from the reference's Post_processing directory (given with --ref) and
restates only the trajectory loop.  With --interp the actions after the first
come from the reference's own ``get_interpolated_action`` (the script's
``with_policy_interp=True`` branch, :483-486 with :174-198 and the
interpolation helpers :37-171); plot_e2eGPU_policy imports matplotlib, imageio
and cv2 for its plots only, which are absent here, so inert stand-ins for those
modules are put in ``sys.modules`` before importing it (nothing used goes
through them), and its module-level ``gsize`` (set by its ``__main__`` block)
is set to the problem's grid size.  Inputs are the seeded fields of the named problems and
the reference's own solved policies stored in tests/golden/ref_<name>.npz.
Arithmetic follows NumPy's scalar rules of the installed NumPy (2.x: a Python
float with a float32 stays float32); the fixtures record the NumPy version.

    python tests/golden/make_rollout_golden.py --ref <reference>/Post_processing

writes tests/golden/rollout_<name>.npz (start cells, per-realisation outcome,
travel time, energies, final state); with --interp rollout_interp_<name>.npz.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

NAMES = ["t_time", "t_custom", "c1"]
STARTS = {"t_time": [(8, 12), (3, 3), (14, 1)], "t_custom": [(10, 17), (2, 2)], "c1": [(25, 47), (10, 5)]}


def rollout_reference(grid_world, prob, fields, policy, start, interp=None):
    """The trajectory loop of plot_exact_trajectory_set_DP (:433-474) around the
    reference's Grid.move_exact, for every realisation."""
    params = prob.prob_params()
    gsize = int(params[0])
    dx, dy = params[16], params[17]
    xs = [(dx / 2) + (i * dx) for i in range(gsize)]   # setup_grid.py Test_grid branch
    ys = [(dy / 2) + (i * dy) for i in range(gsize)]
    g = grid_world.timeOpt_grid(xs, ys, int(params[12]), params[4], int(params[10]), params[3], start,
                                (int(params[8]), int(params[9])), num_ac_speeds=int(params[14]),
                                num_ac_angles=int(params[15]))
    vel = [fields["u"], fields["v"], fields["ui"], fields["vi"], fields["Yi"]]
    s_mat, mask = fields["s"], fields["mask"]
    nrz = fields["Yi"].shape[1]
    out = {k: [] for k in ("success", "travel_time", "energy_cons", "energy_col", "net_energy", "t", "i", "j")}
    Cf, Cr = 1, 1
    for rzn in range(nrz):
        success = None
        energy_cons = energy_col = net_energy = 0
        travel_time = 0
        g.set_state(g.start_state)
        t, i, j = g.start_state
        a = g.actions[int(policy[j + gsize * i + gsize * gsize * t])]
        for _ in range(g.nt):
            if success is None:
                vx = vel[0][t, i, j] + np.matmul(vel[2][t, :, i, j], vel[4][t, rzn, :])
                vy = vel[1][t, i, j] + np.matmul(vel[3][t, :, i, j], vel[4][t, rzn, :])
                rad1 = s_mat[t, i, j]
                g.move_exact(a, vx, vy)
                (t, i, j) = g.current_state()
                rad2 = s_mat[t, i, j]
                travel_time += 1
                energy_cons += (Cf * a[0]) ** 2
                energy_col += (Cr * (rad2 + rad1) / 2)
                net_energy += (Cf * (a[0] ** 2)) - (Cr * (rad2 + rad1) / 2)
            if g.if_edge_state((i, j)) or mask[t, i, j] == 1:
                success = False
            if (not g.is_terminal()) and g.if_within_actionable_time() and success is None:
                if interp is not None:
                    a = interp(g)
                else:
                    a = g.actions[int(policy[j + gsize * i + gsize * gsize * t])]
            elif g.is_terminal():
                success = True
            else:
                success = False
        out["success"].append(-1 if success is None else int(success))
        out["travel_time"].append(travel_time)
        out["energy_cons"].append(energy_cons)
        out["energy_col"].append(energy_col)
        out["net_energy"].append(net_energy)
        out["t"].append(t)
        out["i"].append(i)
        out["j"].append(j)
    return {"success": np.array(out["success"], np.int8), "travel_time": np.array(out["travel_time"], np.int32),
            "energy_cons": np.array(out["energy_cons"], np.float64),
            "energy_col": np.array(out["energy_col"], np.float64),
            "net_energy": np.array(out["net_energy"], np.float64),
            "final_tij": np.stack([out["t"], out["i"], out["j"]], 1).astype(np.int32)}


class _Inert:
    """Stand-in for the plotting modules: every attribute and call returns itself."""

    def __getattr__(self, name):
        return self

    def __call__(self, *a, **k):
        return self


def load_policy_script():
    import types
    mpl = types.ModuleType("matplotlib")
    for sub in ("pyplot", "colors", "cm"):
        setattr(mpl, sub, _Inert())
        sys.modules.setdefault(f"matplotlib.{sub}", getattr(mpl, sub))
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("imageio", _Inert())
    sys.modules.setdefault("cv2", _Inert())
    import plot_e2eGPU_policy  # noqa: E402
    return plot_e2eGPU_policy


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference's Post_processing directory")
    ap.add_argument("--interp", action="store_true", help="actions from get_interpolated_action")
    ap.add_argument("names", nargs="*", default=NAMES)
    args = ap.parse_args()
    sys.path.insert(0, os.path.abspath(args.ref))
    cwd = os.getcwd()
    os.chdir(args.ref)  # its modules import siblings relative to that directory
    import grid_world   # noqa: E402
    pp = load_policy_script() if args.interp else None
    os.chdir(cwd)
    from tests.helpers import golden, problem
    for name in args.names:
        prob, fields = problem(name)
        policy = golden(name)["policy"].astype(np.int64)
        interp = None
        if pp is not None:
            pp.gsize = int(prob.prob_params()[0])
            policy_1d = policy.reshape(-1, 1)
            interp = lambda g, pol=policy_1d: pp.get_interpolated_action(pol, g)  # noqa: E731
        res = {}
        for k, st in enumerate(STARTS[name]):
            r = rollout_reference(grid_world, prob, fields, policy, st, interp=interp)
            for key, v in r.items():
                res[f"{key}_{k}"] = v
        fname = f"rollout_interp_{name}.npz" if args.interp else f"rollout_{name}.npz"
        np.savez_compressed(os.path.join(HERE, fname), starts=np.array(STARTS[name], np.int32),
                            numpy_version=np.array(np.__version__), **res)
        succ = [float(np.mean(res[f"success_{k}"] == 1)) for k in range(len(STARTS[name]))]
        print(name, "success rates", succ)


if __name__ == "__main__":
    main()
