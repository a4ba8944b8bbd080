"""Environment generator: the reference's double-gyre + westward-cloud fields on the GPU.

``build_environment_DG_with_westward_clouds`` has the argument list of the
reference's function (src/data_input/build_environment_DG_with_westward_clouds.py:
510-590) and produces the same ten arrays (returned, and written as the
reference's .npy files when ``out_dir`` is given); the work runs in
``e2e_env_generate`` of libe2edp.so.  The one host-side step is the
interpolation table: the reference interpolates with scipy's griddata
('linear': a Delaunay triangulation of the coarse cell centres and barycentric
weights), and this module builds that triangulation with the same scipy call so
that the GPU evaluates identical triangles and weights.
"""
from __future__ import annotations

import ctypes as C
import os
from math import pi
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import check, lib

FILES = ("all_u_mat", "all_v_mat", "all_ui_mat", "all_vi_mat", "all_Yi", "all_phi_mat", "all_phi_i_mat",
         "all_phi_Yi_mat", "all_s_mat", "obstacle_mask")


def grid_ticks(gsize: int, dxy: float):
    """Cell centres (0.5 + i) dxy (get_xs_ys, :127-128)."""
    return [(0.5 + i) * dxy for i in range(gsize)]


def interp_table(init_gsize: int, dxy: float, degree: int) -> Tuple[np.ndarray, np.ndarray]:
    """Triangle vertices (G*G x 3, int32, -1 outside the hull) and barycentric
    weights (G*G x 3, float64) of every fine-grid point in the Delaunay
    triangulation of the coarse cell centres, for griddata 'linear'
    (interpolate_data_t, :265-283).  The simplex search is scipy's own
    (Delaunay.find_simplex walks from the previous point's simplex, as the
    interpolator does); the weights repeat scipy's barycentric arithmetic
    (c_i = sum_j T_ij (x_j - r_j) left to right, c_2 = 1 - c_0 - c_1)."""
    from scipy.spatial import Delaunay

    xs = grid_ticks(init_gsize, dxy)
    xgrid, ygrid = np.meshgrid(xs, np.flip(xs))
    points = np.empty((init_gsize * init_gsize, 2))
    points[:, 0] = xgrid.flatten()
    points[:, 1] = ygrid.flatten()
    nx = grid_ticks(init_gsize * degree, dxy / degree)
    nxg, nyg = np.meshgrid(nx, np.flip(nx))
    xi = np.ascontiguousarray(np.stack([nxg.ravel(), nyg.ravel()], axis=1), dtype=np.float64)
    tri = Delaunay(points)
    simp = tri.find_simplex(xi)
    inside = simp >= 0
    T = tri.transform[np.where(inside, simp, 0)]
    d0 = xi[:, 0] - T[:, 2, 0]
    d1 = xi[:, 1] - T[:, 2, 1]
    c0 = (0.0 + T[:, 0, 0] * d0) + T[:, 0, 1] * d1
    c1 = (0.0 + T[:, 1, 0] * d0) + T[:, 1, 1] * d1
    c2 = (1.0 - c0) - c1
    vert = tri.simplices[np.where(inside, simp, 0)].astype(np.int32)
    vert[~inside] = -1
    wgt = np.stack([c0, c1, c2], axis=1)
    wgt[~inside] = 0.0
    return np.ascontiguousarray(vert), np.ascontiguousarray(wgt)


def env_params(init_gsize, nt, dt, dxy, A, A_sc, eps, n_wsamples, w_range, wx, interpolate_degree, n_modes,
               dyn_obstacle_data: Optional[Sequence] = None) -> _lib.EnvParams:
    """The C parameter block; dyn_obstacle_data as the reference's
    (('None',), ('static',) or (upper_row, left_col, width, (speed_x, speed_y), 'dynamic'))."""
    mode, ou, ol, ow, sx, sy = _lib.E2E_OBST_NONE, 0.0, 0.0, 0.0, 0.0, 0.0
    if dyn_obstacle_data is not None:
        kind = dyn_obstacle_data[-1]
        if kind == "static":
            mode = _lib.E2E_OBST_STATIC
        elif kind == "dynamic":
            ou, ol, ow, speed = dyn_obstacle_data[0], dyn_obstacle_data[1], dyn_obstacle_data[2], dyn_obstacle_data[3]
            G = init_gsize * interpolate_degree
            if not (0 < ol < G and 0 < ou < G):  # the reference's assertion (:450)
                raise ValueError("dynamic obstacle must start inside the grid")
            mode, sx, sy = _lib.E2E_OBST_DYNAMIC, float(speed[0]), float(speed[1])
        elif kind != "None":
            raise ValueError(f"unknown obstacle mode {kind!r}")
    return _lib.EnvParams(int(init_gsize), int(nt), int(n_wsamples), int(n_modes), int(interpolate_degree), mode,
                          float(dt), float(dxy), float(A), float(A_sc), float(eps), float(w_range[0]),
                          float(w_range[1]), float(wx), float(ou), float(ol), float(ow), sx, sy)


def build_environment_DG_with_westward_clouds(init_gsize, nt, dt, dxy, A, A_sc, eps, op_nrzns, n_wsamples, w_range,
                                              wx, interpolate_degree, n_modes, dyn_obstacle_data=None,
                                              out_dir: Optional[str] = None, device: bool = False,
                                              stream=None) -> Dict:
    """All fields of the reference generator, computed on the GPU.  Returns a
    dict keyed by the reference's file names (numpy arrays, or CUDA tensors with
    ``device=True``) plus ``svals_vel`` / ``svals_phi`` (nt x n_modes singular
    values) and ``stats``; with ``out_dir`` the .npy files are written there.
    ``op_nrzns`` is accepted for the reference's signature and not used (as there)."""
    del op_nrzns
    if dyn_obstacle_data is None:
        raise ValueError("dyn_obstacle_data is required (the reference reads its last entry)")
    p = env_params(init_gsize, nt, dt, dxy, A, A_sc, eps, n_wsamples, w_range, wx, interpolate_degree, n_modes,
                   dyn_obstacle_data)
    vert, wgt = interp_table(init_gsize, dxy, interpolate_degree)
    G = init_gsize * interpolate_degree
    shapes = {"all_u_mat": (nt, G, G), "all_v_mat": (nt, G, G), "all_ui_mat": (nt, n_modes, G, G),
              "all_vi_mat": (nt, n_modes, G, G), "all_Yi": (nt, n_wsamples, n_modes), "all_phi_mat": (nt, G, G),
              "all_phi_i_mat": (nt, n_modes, G, G), "all_phi_Yi_mat": (nt, n_wsamples, n_modes),
              "all_s_mat": (nt, G, G), "obstacle_mask": (nt, G, G)}
    if device:
        import torch

        out = {k: torch.empty(s, dtype=torch.int32 if k == "obstacle_mask" else torch.float32, device="cuda")
               for k, s in shapes.items()}
        ptr = {k: v.data_ptr() for k, v in out.items()}
        where = _lib.E2E_DEVICE
        sptr = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    else:
        out = {k: np.empty(s, dtype=np.int32 if k == "obstacle_mask" else np.float32) for k, s in shapes.items()}
        ptr = {k: v.ctypes.data for k, v in out.items()}
        where = _lib.E2E_HOST
        sptr = None
    f = _lib.EnvFields(ptr["all_u_mat"], ptr["all_v_mat"], ptr["all_ui_mat"], ptr["all_vi_mat"], ptr["all_Yi"],
                       ptr["all_phi_mat"], ptr["all_phi_i_mat"], ptr["all_phi_Yi_mat"], ptr["all_s_mat"],
                       ptr["obstacle_mask"])
    sv = np.empty((2, nt, n_modes), np.float64)
    st = _lib.EnvStats()
    check(lib().e2e_env_generate(C.byref(p), vert.ctypes.data, wgt.ctypes.data, where, C.byref(f), sv.ctypes.data,
                                 C.byref(st), sptr))
    if out_dir is not None:
        os.makedirs(out_dir, exist_ok=True)
        for k in FILES:
            a = out[k].cpu().numpy() if device else out[k]
            np.save(os.path.join(out_dir, k + ".npy"), a)
    out["svals_vel"] = sv[0]
    out["svals_phi"] = sv[1]
    out["stats"] = {k: getattr(st, k) for k, _ in _lib.EnvStats._fields_}
    return out


def reference_defaults() -> Dict:
    """The parameter block written out in the reference script (:494-507)."""
    init_gsize, nt = 25, 10
    return dict(init_gsize=init_gsize, nt=nt, dt=10 / nt, dxy=2 / init_gsize, A=0.5, A_sc=3, eps=0.1, op_nrzns=10,
                n_wsamples=1000, w_range=(pi / 10, 8 * pi / 10), wx=pi, interpolate_degree=8, n_modes=3)
