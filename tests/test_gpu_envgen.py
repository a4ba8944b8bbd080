"""GPU parity of the environment generator (e2e_env_generate) with the reference's.

tests/golden/env_*.npz hold the arrays the reference's own
build_environment_DG_with_westward_clouds wrote.  Integer and elementwise
outputs (obstacle mask, cloud field) must match bit for bit; means of the
realisations within two float32 ulps (the device's double sin/cos may differ
from the host libm's in the last bit); the rank reduction is an SVD, defined
up to the sign of each mode, so modes and coefficients are compared after
aligning signs, singular values relative to the largest, and the sign-free
products of modes and coefficients (what the builder reads) directly.  At
t = 0 every realisation is the same (sin(w*0) = 0): the centred matrix is
rounding noise, its singular vectors are arbitrary in any implementation, and
only the (tiny) products are compared there.
"""
import os

import numpy as np
import pytest

from e2e_gpu_dp_b200 import envgen
from oracle import envgen as OE

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ["env_a", "env_b", "env_c"]


def _golden(name):
    return np.load(os.path.join(HERE, "golden", f"{name}.npz"))


@pytest.fixture(scope="module")
def generated():
    cache = {}

    def get(name):
        if name not in cache:
            z = _golden(name)
            cfg = OE.config_from_golden(z)
            out = envgen.build_environment_DG_with_westward_clouds(op_nrzns=10, **cfg)
            st = int(z["grid_stride"])
            sub = {k: (out[k][..., ::st, ::st] if k not in ("all_Yi", "all_phi_Yi_mat") else out[k])
                   for k in OE.FILES}
            cache[name] = (z, cfg, out, sub)
        return cache[name]

    return get


def _close_f32(a, b, ulps=2):
    tol = ulps * np.spacing(np.maximum(np.abs(a), np.abs(b)).astype(np.float32)).astype(np.float64)
    return np.abs(a.astype(np.float64) - b.astype(np.float64)) <= tol + 1e-30


@pytest.mark.parametrize("name", NAMES)
def test_mask_and_cloud_bit_exact(generated, name):
    z, cfg, out, sub = generated(name)
    assert np.array_equal(sub["obstacle_mask"], z["obstacle_mask"])
    assert np.array_equal(sub["all_s_mat"], z["all_s_mat"])


@pytest.mark.parametrize("name", NAMES)
def test_means_within_two_ulps(generated, name):
    z, cfg, out, sub = generated(name)
    for k in ("all_u_mat", "all_v_mat", "all_phi_mat"):
        ok = _close_f32(sub[k], z[k])
        assert ok.all(), (k, int((~ok).sum()), float(np.max(np.abs(sub[k] - z[k]))))


def _live_steps(z, key):
    s = z[key]
    return [t for t in range(s.shape[0]) if s[t, 0] > 1e-8 * s[:, 0].max()]


@pytest.mark.parametrize("name", NAMES)
def test_singular_values(generated, name):
    z, cfg, out, sub = generated(name)
    r = cfg["n_modes"]
    for mine, key in ((out["svals_vel"], "svals_vel"), (out["svals_phi"], "svals_phi")):
        for t in _live_steps(z, key):
            ref = z[key][t, :r]
            assert np.max(np.abs(mine[t] - ref)) <= 1e-12 * ref[0], (key, t, mine[t], ref)


@pytest.mark.parametrize("name", NAMES)
def test_modes_and_coefficients_up_to_sign(generated, name):
    z, cfg, out, sub = generated(name)
    r = cfg["n_modes"]
    groups = (("all_Yi", ("all_ui_mat", "all_vi_mat"), "svals_vel"),
              ("all_phi_Yi_mat", ("all_phi_i_mat",), "svals_phi"))
    for ck, mks, sk in groups:
        for t in _live_steps(z, sk):
            for m in range(r):
                c_ref, c_mine = z[ck][t, :, m].astype(np.float64), sub[ck][t, :, m].astype(np.float64)
                sgn = 1.0 if np.dot(c_ref, c_mine) >= 0 else -1.0
                scale = np.max(np.abs(c_ref))
                assert np.max(np.abs(sgn * c_mine - c_ref)) <= 2e-6 * scale, (ck, t, m)
                for mk in mks:
                    a_ref, a_mine = z[mk][t, m].astype(np.float64), sub[mk][t, m].astype(np.float64)
                    assert np.max(np.abs(sgn * a_mine - a_ref)) <= 2e-6 * max(np.max(np.abs(a_ref)), 1e-30), \
                        (mk, t, m)


@pytest.mark.parametrize("name", NAMES)
def test_mode_products_sign_free(generated, name):
    # sum_m ui_m Y_m at every (t, realisation, fine cell): what the builder reads
    z, cfg, out, sub = generated(name)
    for ck, mk in (("all_Yi", "all_ui_mat"), ("all_Yi", "all_vi_mat"), ("all_phi_Yi_mat", "all_phi_i_mat")):
        ref = np.einsum("tkm,tmij->tkij", z[ck].astype(np.float64), z[mk].astype(np.float64))
        mine = np.einsum("tkm,tmij->tkij", sub[ck].astype(np.float64), sub[mk].astype(np.float64))
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(mine - ref)) <= 1e-5 * scale, (ck, mk, float(np.max(np.abs(mine - ref))), scale)


@pytest.mark.parametrize("name", NAMES)
def test_range_finder_certifies_every_step(generated, name):
    # the first range finder (n_modes + 10 columns, two power iterations) is
    # certified on every step: by its residual where the realisations differ,
    # as rounding noise of the centring at t = 0; none is re-run enlarged
    z, cfg, out, sub = generated(name)
    assert out["stats"]["full_svds"] == 0, out["stats"]


def test_range_finder_spanning_the_whole_side():
    # a 2 x 2 coarse grid: the velocity matrix has 8 columns and the scalar one
    # 4, fewer than n_modes + 10, so the range finder takes all of them; the
    # singular values and the products mode x coefficient match the CPU
    # restatement (numpy's SVD)
    cfg = dict(init_gsize=2, nt=3, dt=0.5, dxy=1.0, A=0.5, A_sc=3.0, eps=0.1, n_wsamples=16,
               w_range=(np.pi / 10, 8 * np.pi / 10), wx=np.pi, interpolate_degree=2, n_modes=3,
               dyn_obstacle_data=("None",))
    out = envgen.build_environment_DG_with_westward_clouds(op_nrzns=10, **cfg)
    ref = OE.generate(**cfg)
    assert out["stats"]["full_svds"] == 0, out["stats"]
    r = cfg["n_modes"]
    for key in ("svals_vel", "svals_phi"):
        s_ref = ref[key][:, :r]
        for t in range(cfg["nt"]):
            if s_ref[t, 0] > 1e-8 * s_ref[:, 0].max():
                assert np.max(np.abs(out[key][t] - s_ref[t])) <= 1e-12 * s_ref[t, 0], (key, t)
    for ck, mk in (("all_Yi", "all_ui_mat"), ("all_Yi", "all_vi_mat"), ("all_phi_Yi_mat", "all_phi_i_mat")):
        a = np.einsum("tkm,tmij->tkij", ref[ck].astype(np.float64), ref[mk].astype(np.float64))
        b = np.einsum("tkm,tmij->tkij", out[ck].astype(np.float64), out[mk].astype(np.float64))
        assert np.max(np.abs(a - b)) <= 1e-5 * np.max(np.abs(a)), (ck, mk)


def test_bad_interpolation_table_is_an_error():
    # a caller-built table whose vertex indices leave the coarse grid: the kernel
    # skips those reads, and the call reports E2E_ERR_INVALID
    import ctypes as C

    from e2e_gpu_dp_b200 import _lib
    from e2e_gpu_dp_b200._lib import E2EError
    z = _golden("env_a")
    cfg = OE.config_from_golden(z)
    p = envgen.env_params(**{k: v for k, v in cfg.items()})
    vert, wgt = envgen.interp_table(cfg["init_gsize"], cfg["dxy"], cfg["interpolate_degree"])
    inside = np.flatnonzero(vert[:, 0] >= 0)
    vert[inside[0], 1] = cfg["init_gsize"] ** 2  # one past the last coarse cell
    G, nt, r, nws = cfg["init_gsize"] * cfg["interpolate_degree"], cfg["nt"], cfg["n_modes"], cfg["n_wsamples"]
    arrs = [np.empty((nt, G, G), np.float32) for _ in range(2)] + [np.empty((nt, r, G, G), np.float32) for _ in range(2)]
    arrs += [np.empty((nt, nws, r), np.float32), np.empty((nt, G, G), np.float32), np.empty((nt, r, G, G), np.float32),
             np.empty((nt, nws, r), np.float32), np.empty((nt, G, G), np.float32), np.empty((nt, G, G), np.int32)]
    f = _lib.EnvFields(*[a.ctypes.data for a in arrs])
    rc = _lib.lib().e2e_env_generate(C.byref(p), vert.ctypes.data, wgt.ctypes.data, _lib.E2E_HOST, C.byref(f),
                                     None, None, None)
    assert rc == _lib.E2E_ERR_INVALID
    with pytest.raises(E2EError):
        _lib.check(rc)


def test_device_outputs_equal_host_outputs(generated):
    torch = pytest.importorskip("torch")
    z, cfg, out, sub = generated("env_a")
    dev = envgen.build_environment_DG_with_westward_clouds(op_nrzns=10, device=True, **cfg)
    torch.cuda.synchronize()
    for k in OE.FILES:
        assert np.array_equal(dev[k].cpu().numpy(), out[k]), k


def test_generated_fields_drive_the_planner(generated):
    # the generated files are the builder's inputs: plan on them end to end
    from e2e_gpu_dp_b200 import api
    from e2e_gpu_dp_b200.problem import Problem

    cfg = dict(init_gsize=10, nt=6, dt=0.5, dxy=1.0, A=0.5, A_sc=3.0, eps=0.1, n_wsamples=64,
               w_range=(np.pi / 10, 8 * np.pi / 10), wx=np.pi, interpolate_degree=3, n_modes=3,
               dyn_obstacle_data=(10, 12, 3, (0.5, 0.0), "dynamic"))
    env = envgen.build_environment_DG_with_westward_clouds(op_nrzns=10, **cfg)
    G = 30
    prob = Problem(gsize=G, nt=cfg["nt"], nrzns=cfg["n_wsamples"], nmodes=cfg["n_modes"], num_ac_angles=8,
                   F=1.0, dt=1.0, dx=1.0, dy=1.0, i_term=15, j_term=25, neighb_gsize=9, prob_name="env_gen")
    fields = {"u": env["all_u_mat"], "v": env["all_v_mat"], "ui": env["all_ui_mat"], "vi": env["all_vi_mat"],
              "Yi": env["all_Yi"], "s": env["all_s_mat"], "mask": env["obstacle_mask"]}
    m = api.build_model(prob, fields)
    V, pi, st = m.solve(method="layered")
    Vf, pif, _ = api.build_solve(prob, fields)
    m.free()
    assert st["residual"] == 0.0
    assert np.array_equal(V, Vf) and np.array_equal(pi, pif)
    assert np.all(np.isfinite(V)) and pi.min() >= -1 and pi.max() < prob.num_actions
