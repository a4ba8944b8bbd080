"""CPU restatement of the reference's environment generator (test infrastructure only).

Follows src/data_input/build_environment_DG_with_westward_clouds.py:
realisations (DG_velocity_field.vx_vy / phi / sample_w, :130-184) with Python
float arithmetic in the reference's evaluation order; per-time mean over the
samples and rank reduction of the centred matrix by np.linalg.svd
(compute_modes_and_coeffs / compute_phi_modes_and_coefs / rank_reduction,
:194-262); reshape (:265-292); scipy griddata 'linear' to the refined grid
(:294-329); the cloud field (DG_scalar_field, :20-98) and fill_obstacles
(:441-468).  Pinned bit for bit against tests/golden/env_*.npz, which the
reference's own function produced (tests/golden/make_env_golden.py).
Pure-Python loops: small grids only.
"""
from math import cos, floor, pi, sin
from typing import Dict, Sequence

import numpy as np

FILES = ("all_u_mat", "all_v_mat", "all_ui_mat", "all_vi_mat", "all_Yi", "all_phi_mat", "all_phi_i_mat",
         "all_phi_Yi_mat", "all_s_mat", "obstacle_mask")


def ticks(g: int, dxy: float):
    return [(0.5 + i) * dxy for i in range(g)]


def realisations(g, nt, dt, dxy, A, eps, wx, nws, w_range):
    """R (nt, nws, 2 g^2): vx then vy; phi (nt, nws, g^2); float64."""
    wy = 0.5 * pi
    xs = ticks(g, dxy)
    ys = xs
    n = g * g
    R = np.empty((nt, nws, 2 * n))
    P = np.empty((nt, nws, n))
    for ti in range(nt):
        t = ti * dt
        for k in range(nws):
            w = w_range[0] + (k / (nws - 1)) * (w_range[1] - w_range[0])
            s = sin(w * t)
            for i in range(g):
                y = ys[g - 1 - i]
                for j in range(g):
                    x = xs[j]
                    f = eps * s * (x ** 2) + (1 - 2 * eps * s) * x
                    fx = (2 * eps * s * (x - 1)) + 1
                    c = g * i + j
                    R[ti, k, c] = -(0.5 * A * pi * sin(wx * f) * cos(wy * y))
                    R[ti, k, n + c] = A * pi * sin(wy * y) * fx * cos(wx * f)
                    P[ti, k, c] = A * sin(pi * f) * sin(wy * y)
    return R, P


def reduce_rank(X3: np.ndarray, r: int):
    """Per time: mean over samples, SVD of the centred matrix, C = U_r diag(s_r),
    M = Vh_r (float32), the mean (float64) and all singular values."""
    nt, nws, ncols = X3.shape
    mean = X3.mean(axis=1)
    C = np.empty((nt, nws, r), np.float32)
    M = np.empty((nt, r, ncols), np.float32)
    S = []
    for t in range(nt):
        u, s, vh = np.linalg.svd(X3[t] - mean[t])
        C[t] = np.matmul(u[:, :r], np.diag(s[:r]))
        M[t] = vh[:r]
        S.append(s)
    return C, M, mean, np.stack(S)


def interpolate(field: np.ndarray, g: int, dxy: float, d: int) -> np.ndarray:
    from scipy.interpolate import griddata

    xs = ticks(g, dxy)
    xg, yg = np.meshgrid(xs, np.flip(xs))
    pts = np.stack([xg.flatten(), yg.flatten()], axis=1)
    nx = ticks(g * d, dxy / d)
    nxg, nyg = np.meshgrid(nx, np.flip(nx))
    return griddata(pts, field.flatten(), (nxg, nyg), method="linear")


def cloud(G: int, nt: int, dxy_f: float, A_sc: float) -> np.ndarray:
    xs = ticks(G, dxy_f)
    l = xs[-1] / 2
    dom = xs[-1] + dxy_f
    out = np.empty((nt, G, G), np.float32)
    for t in range(nt):
        T = t * 1 / 2
        for j in range(G):
            x = xs[j]
            xt = x + (T * dxy_f)
            if xt <= l:
                f = 1
            elif l < xt < l + (0.2 * dom):
                f = 1 + ((1 - 0) / (-0.2 * dom)) * (x - (l - T * dxy_f))
            else:
                f = 0
            out[t, :, j] = A_sc * f
    return out


def obstacles(G: int, nt: int, spec: Sequence) -> np.ndarray:
    m = np.zeros((nt, G, G), np.int32)
    mode = spec[-1]
    if mode == "static":
        m[:, int(0.4 * G):int(0.5 * G), int(0.5 * G):int(0.6 * G)] = 1
    elif mode == "dynamic":
        ru_i, cl_i, width, speed = spec[0], spec[1], spec[2], spec[3]
        for t in range(nt):
            cl = floor(cl_i + t * speed[0])
            cr = int(cl + width)
            ru = floor(ru_i + t * speed[1])
            rd = int(ru + width)
            if 0 < cl < G - 1 and 0 < cr < G - 1 and 0 < ru < G - 1 and 0 < rd < G - 1:
                m[t, ru:rd, cl:cr] = 1
    return m


def generate(init_gsize, nt, dt, dxy, A, A_sc, eps, n_wsamples, w_range, wx, interpolate_degree, n_modes,
             dyn_obstacle_data) -> Dict[str, np.ndarray]:
    g, d, r = init_gsize, interpolate_degree, n_modes
    n, G = g * g, g * d
    R, P = realisations(g, nt, dt, dxy, A, eps, wx, n_wsamples, w_range)
    C, M, mean, Sv = reduce_rank(R, r)
    Cp, Mp, meanp, Sp = reduce_rank(P, r)
    # all_u_mat / all_v_mat and the modes are float32 arrays, all_phi_mat is
    # float64 (np.empty without a dtype, :271) and is interpolated unrounded
    coarse = {"u": mean[:, :n].astype(np.float32), "v": mean[:, n:].astype(np.float32),
              "phi": meanp, "ui": M[:, :, :n], "vi": M[:, :, n:], "phi_i": Mp}
    out = {}
    for key, name in (("u", "all_u_mat"), ("v", "all_v_mat"), ("phi", "all_phi_mat")):
        out[name] = np.stack([interpolate(coarse[key][t].reshape(g, g), g, dxy, d) for t in range(nt)]
                             ).astype(np.float32)
    for key, name in (("ui", "all_ui_mat"), ("vi", "all_vi_mat"), ("phi_i", "all_phi_i_mat")):
        out[name] = np.stack([[interpolate(coarse[key][t, m].reshape(g, g), g, dxy, d) for m in range(r)]
                              for t in range(nt)]).astype(np.float32)
    out["all_Yi"] = C
    out["all_phi_Yi_mat"] = Cp
    for k in list(out):
        out[k] = np.nan_to_num(out[k])
    out["all_s_mat"] = cloud(G, nt, dxy / d, A_sc)
    out["obstacle_mask"] = obstacles(G, nt, dyn_obstacle_data)
    out["R_vel"], out["R_phi"], out["svals_vel"], out["svals_phi"] = R, P, Sv, Sp
    return out


def config_from_golden(z) -> Dict:
    p = z["params"]
    import ast
    return dict(init_gsize=int(p[0]), nt=int(p[1]), dt=float(p[2]), dxy=float(p[3]), A=float(p[4]),
                A_sc=float(p[5]), eps=float(p[6]), n_wsamples=int(p[7]), w_range=(float(p[8]), float(p[9])),
                wx=float(p[10]), interpolate_degree=int(p[11]), n_modes=int(p[12]),
                dyn_obstacle_data=ast.literal_eval(str(z["obstacle"])))
