"""Golden vectors of the reference's environment generator.

Runs ``build_environment_DG_with_westward_clouds`` of the reference
(src/data_input/build_environment_DG_with_westward_clouds.py:510-590) itself on
small configurations and stores every array it saves (the eight velocity /
scalar-mode files and all_s_mat, obstacle_mask), plus the singular values of
each time step's centred realisation matrices (``compute_modes_and_coeffs``,
``compute_phi_modes_and_coefs``, :209-262).  The module imports matplotlib and
imageio for its plotting helpers only; they are absent here, so this script
puts inert stand-ins for those two modules in ``sys.modules`` before importing
it (nothing it saves goes through them).  numpy, scipy (griddata) are the real
libraries.

    python tests/golden/make_env_golden.py --ref <reference>/src/data_input

writes tests/golden/env_<name>.npz.
"""
from __future__ import annotations

import argparse
import contextlib
import importlib.util
import io
import os
import sys
import tempfile
import types
from math import pi

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# name -> keyword arguments of build_environment_DG_with_westward_clouds
CONFIGS = {
    # interpolation x2, fewer samples than 2*n (Gram of the sample side), dynamic obstacle
    "env_a": dict(init_gsize=6, nt=3, dt=10 / 3, dxy=2 / 6, A=0.5, A_sc=3.0, eps=0.1, op_nrzns=10,
                  n_wsamples=24, w_range=(pi / 10, 8 * pi / 10), wx=pi, interpolate_degree=2, n_modes=3,
                  dyn_obstacle_data=(3, 4, 2, (0.5, 0.25), "dynamic")),
    # no interpolation, more samples than 2*n (Gram of the grid side), static obstacle
    "env_b": dict(init_gsize=4, nt=4, dt=0.5, dxy=0.5, A=0.5, A_sc=3.0, eps=0.1, op_nrzns=10,
                  n_wsamples=40, w_range=(pi / 10, 8 * pi / 10), wx=pi, interpolate_degree=1, n_modes=4,
                  dyn_obstacle_data=("static",)),
    # the reference's default grid (25 x 25, 8x interpolation to 200 x 200) at three time steps
    # (the reference asserts n_modes <= min(nt, n_wsamples, 2 n), :213)
    "env_c": dict(init_gsize=25, nt=3, dt=1.0, dxy=2 / 25, A=0.5, A_sc=3.0, eps=0.1, op_nrzns=10,
                  n_wsamples=60, w_range=(pi / 10, 8 * pi / 10), wx=pi, interpolate_degree=8, n_modes=3,
                  dyn_obstacle_data=("None",)),
}

FILES = ["all_u_mat", "all_v_mat", "all_ui_mat", "all_vi_mat", "all_Yi", "all_phi_mat", "all_phi_i_mat",
         "all_phi_Yi_mat", "all_s_mat", "obstacle_mask"]


class _Inert:
    """Stand-in for the plotting modules: every attribute and call returns itself."""

    def __getattr__(self, name):
        return self

    def __call__(self, *a, **k):
        return self


def load_reference(ref_dir: str):
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = _Inert()
    sys.modules.setdefault("matplotlib", mpl)
    sys.modules.setdefault("matplotlib.pyplot", mpl.pyplot)
    sys.modules.setdefault("imageio", _Inert())
    path = os.path.join(ref_dir, "build_environment_DG_with_westward_clouds.py")
    spec = importlib.util.spec_from_file_location("ref_env_generator", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def run(mod, cfg):
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as d:
        os.chdir(d)
        try:
            with contextlib.redirect_stdout(io.StringIO()):
                mod.build_environment_DG_with_westward_clouds(**cfg)
                out = {k: np.load(k + ".npy") for k in FILES}
                # singular values of the centred realisation matrices, per time step
                dg = mod.DG_velocity_field(cfg["init_gsize"], cfg["nt"], cfg["dt"], cfg["dxy"], cfg["A"],
                                           cfg["eps"], cfg["wx"], 0.5 * pi, cfg["op_nrzns"],
                                           cfg["n_wsamples"], cfg["w_range"], cfg["interpolate_degree"])
                Rx, Ry, phi = dg.generate_R()
                R = np.concatenate((Rx, Ry), axis=2)
                X = R - R.mean(axis=1, keepdims=True)
                P = phi - phi.mean(axis=1, keepdims=True)
                out["svals_vel"] = np.stack([np.linalg.svd(X[t], compute_uv=False) for t in range(cfg["nt"])])
                out["svals_phi"] = np.stack([np.linalg.svd(P[t], compute_uv=False) for t in range(cfg["nt"])])
                out["R_vel"] = R
                out["R_phi"] = phi
        finally:
            os.chdir(cwd)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference's src/data_input directory")
    ap.add_argument("names", nargs="*", default=list(CONFIGS))
    args = ap.parse_args()
    mod = load_reference(os.path.abspath(args.ref))
    for name in args.names:
        cfg = CONFIGS[name]
        out = run(mod, cfg)
        params = np.array([cfg["init_gsize"], cfg["nt"], cfg["dt"], cfg["dxy"], cfg["A"], cfg["A_sc"], cfg["eps"],
                           cfg["n_wsamples"], cfg["w_range"][0], cfg["w_range"][1], cfg["wx"],
                           cfg["interpolate_degree"], cfg["n_modes"]], np.float64)
        stride = 1
        if name == "env_c":  # keep the fixture small: no realisation matrices, every 5th row and column
            out.pop("R_vel")
            out.pop("R_phi")
            stride = 5
            for k in FILES:
                if k not in ("all_Yi", "all_phi_Yi_mat"):
                    out[k] = np.ascontiguousarray(out[k][..., ::stride, ::stride])
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), params=params,
                            obstacle=np.array(repr(cfg["dyn_obstacle_data"])), grid_stride=np.array(stride),
                            numpy_version=np.array(np.__version__), **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
