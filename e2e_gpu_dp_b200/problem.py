"""Problem description, the ``prob_params`` slot layout, action tables and the
seeded synthetic environment generator.

The reference takes its problem definition from a compile-time header
(``src/input_to_build_model.h:1-48``) that ``main`` includes inside its body
(``src/build_model.cu:932``) and forwards to the device as a 32-float vector
(``src/build_model.cu:1032-1055``), which is also saved as ``prob_params.npy``
for the downstream consumers.  :class:`Problem` carries the same fields at
run time and reproduces that slot layout exactly (:meth:`Problem.prob_params`).

The reference ships no input data (its ``data_input/`` is absent), so the
velocity fields here are synthetic and seeded: a double-gyre mean flow plus
low-frequency Fourier modes with Gaussian coefficients, written in the
reference's on-disk layout (``src/build_model.cu:978-985``):

==============  ======================  =======
file            shape                   dtype
==============  ======================  =======
all_u_mat       (nt, g, g)              float32
all_v_mat       (nt, g, g)              float32
all_ui_mat      (nt, nmodes, g, g)      float32
all_vi_mat      (nt, nmodes, g, g)      float32
all_Yi          (nt, nrzns, nmodes)     float32
all_s_mat       (nt, g, g)              float32
obstacle_mask   (nt, g, g)              int32
==============  ======================  =======
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Dict, Optional, Tuple

import numpy as np

REWARD_TYPES = {"time": 0, "energy1": 1, "energy2": 2, "energy3": 3, "custom1": 4}
FIELD_NAMES = ("u", "v", "ui", "vi", "Yi", "s", "mask")
FIELD_FILES = {
    "u": "all_u_mat.npy",
    "v": "all_v_mat.npy",
    "ui": "all_ui_mat.npy",
    "vi": "all_vi_mat.npy",
    "Yi": "all_Yi.npy",
    "s": "all_s_mat.npy",
    "mask": "obstacle_mask.npy",
}


@dataclasses.dataclass
class Problem:
    """Run-time twin of the reference's config header.

    Field meanings follow ``src/input_to_build_model.h``; the slot numbers in
    the comments are those of ``prob_params`` (``src/build_model.cu:1033-1055``).
    """

    gsize: int                      # slot 0
    nt: int                         # slot 10
    nrzns: int                      # slot 2
    nmodes: int                     # slot 7
    num_ac_speeds: int = 1          # slot 14
    num_ac_angles: int = 8          # slot 15
    F: float = 1.0                  # slot 3 (max vehicle speed)
    dt: float = 1.0                 # slot 4
    dx: float = 1.0                 # slot 16
    dy: float = 1.0                 # slot 17
    r_outbound: float = -100.0      # slot 5
    r_terminal: float = 100.0       # slot 6
    i_term: int = 0                 # slot 8 (top-left row of the terminal subgrid)
    j_term: int = 0                 # slot 9
    term_subgrid_size: int = 1      # slot 12
    neighb_gsize: int = 21          # slot 18 (m, odd, <= gsize)
    prob_type: str = "time"         # slot 13 via REWARD_TYPES
    alpha: float = 0.0              # slot 19
    is_stationary: int = 0          # slot 11
    prob_name: str = "synthetic"

    @property
    def num_actions(self) -> int:
        return self.num_ac_speeds * self.num_ac_angles

    @property
    def reward_type(self) -> int:
        return REWARD_TYPES[self.prob_type]

    @property
    def ncells(self) -> int:
        return self.gsize * self.gsize

    @property
    def ns(self) -> int:
        return self.ncells * self.nt

    @property
    def x0(self) -> float:
        return float(np.float32(self.dx) / np.float32(2))

    @property
    def y0(self) -> float:
        return float(np.float32(self.dy) / np.float32(2))

    def validate(self) -> None:
        m = self.neighb_gsize
        if self.gsize < 2 or self.nt < 2:
            raise ValueError("gsize and nt must be >= 2")
        if m % 2 != 1 or m > self.gsize:
            raise ValueError("neighb_gsize must be odd and <= gsize (src/build_model.cu:1027-1028)")
        if self.prob_type not in REWARD_TYPES:
            raise ValueError(f"unknown prob_type {self.prob_type}")
        if not (0 <= self.i_term < self.gsize and 0 <= self.j_term < self.gsize):
            raise ValueError("terminal cell outside the grid")

    def prob_params(self) -> np.ndarray:
        """The 32-float vector of ``src/build_model.cu:1032-1055`` (slots 20-31 = -9999)."""
        p = np.full(32, -9999.0, dtype=np.float32)
        p[0] = self.gsize
        p[1] = self.num_actions
        p[2] = self.nrzns
        p[3] = self.F
        p[4] = self.dt
        p[5] = self.r_outbound
        p[6] = self.r_terminal
        p[7] = self.nmodes
        p[8] = self.i_term
        p[9] = self.j_term
        p[10] = self.nt
        p[11] = self.is_stationary
        p[12] = self.term_subgrid_size
        p[13] = self.reward_type
        p[14] = self.num_ac_speeds
        p[15] = self.num_ac_angles
        p[16] = self.dx
        p[17] = self.dy
        p[18] = self.neighb_gsize
        p[19] = self.alpha
        return p

    @classmethod
    def from_prob_params(cls, p, prob_name: str = "synthetic") -> "Problem":
        p = np.asarray(p, dtype=np.float32).reshape(-1)
        inv = {v: k for k, v in REWARD_TYPES.items()}
        return cls(
            gsize=int(p[0]), nt=int(p[10]), nrzns=int(p[2]), nmodes=int(p[7]),
            num_ac_speeds=int(p[14]), num_ac_angles=int(p[15]), F=float(p[3]),
            dt=float(p[4]), dx=float(p[16]), dy=float(p[17]), r_outbound=float(p[5]),
            r_terminal=float(p[6]), i_term=int(p[8]), j_term=int(p[9]),
            term_subgrid_size=int(p[12]), neighb_gsize=int(p[18]),
            prob_type=inv[int(p[13])], alpha=float(p[19]), is_stationary=int(p[11]),
            prob_name=prob_name,
        )

    def grid_ticks(self) -> Tuple[np.ndarray, np.ndarray]:
        """Cell-centre coordinates ``xs[i] = x0 + i*dx`` in float32 arithmetic
        (``define_xs_or_ys``, ``src/build_model.cu:1395-1399``)."""
        i = np.arange(self.gsize, dtype=np.float32)
        xs = np.float32(self.x0) + i * np.float32(self.dx)
        ys = np.float32(self.y0) + i * np.float32(self.dy)
        return xs.astype(np.float32), ys.astype(np.float32)

    def actions(self) -> Tuple[np.ndarray, np.ndarray]:
        """(speed, angle) per action index ``j + num_ac_angles*i``.

        Angles are ``j*(2*pi)/n`` evaluated in double and stored as float
        (``populate_ac_angles``, ``src/build_model.cu:1403-1408``); speeds are
        ``Fmax`` for one speed, else ``(i+1)*Fmax/n`` in float
        (``populate_ac_speeds``, ``src/build_model.cu:1412-1434``).
        """
        n = self.num_ac_angles
        angles = np.array([np.float32(j * (2 * math.pi) / n) for j in range(n)], dtype=np.float32)
        if self.num_ac_speeds == 1:
            speeds = np.array([self.F], dtype=np.float32)
        else:
            delF = np.float32(np.float32(self.F) / np.float32(self.num_ac_speeds))
            speeds = np.array([np.float32(np.float32(i + 1) * delF)
                               for i in range(self.num_ac_speeds)], dtype=np.float32)
        sp = np.repeat(speeds, n).astype(np.float32)
        an = np.tile(angles, self.num_ac_speeds).astype(np.float32)
        return sp, an

    def prob_specs(self) -> str:
        """Directory token of ``get_prob_name`` (``src/build_model.cu:658-672``)."""
        return (f"a{self.num_ac_speeds}x{self.num_ac_angles}_i{self.i_term}_j{self.j_term}"
                f"_ref{self.term_subgrid_size}")

    def reference_header(self, bdimx: int = 64) -> str:
        """Text of a config header with the variable set that the reference's
        ``main`` expects from ``input_to_build_model.h`` (the header is the
        reference's configuration interface, so the names and types must match)."""
        def f(x):
            return repr(float(x)) + "f"
        lines = [
            "// generated problem configuration",
            f'std::string prob_type = "{self.prob_type}";',
            f'std::string prob_name = "{self.prob_name}";',
            f"float alpha_header = {f(self.alpha)};",
            f"int32_t nt = {self.nt};",
            f"float dt = {f(self.dt)};",
            f"int32_t gsize = {self.gsize};",
            f"float dx = {f(self.dx)}; float dy = {f(self.dy)};",
            "float x0 = dx/2;",
            "float y0 = dy/2;",
            f"float F = {f(self.F)};",
            f"int num_ac_speeds = {self.num_ac_speeds};",
            f"int num_ac_angles = {self.num_ac_angles};",
            "int32_t num_actions = num_ac_speeds*num_ac_angles;",
            f"int32_t nrzns = {self.nrzns};",
            f"int32_t bDimx = {bdimx};",
            f"float r_outbound = {f(self.r_outbound)};",
            f"float r_terminal = {f(self.r_terminal)};",
            f"int32_t i_term = {self.i_term};",
            f"int32_t j_term = {self.j_term};",
            f"int term_subgrid_size = {self.term_subgrid_size};",
            f"float nmodes = {self.nmodes};",
            f"float neighb_gsize = {self.neighb_gsize};",
            f"int32_t is_stationary = {self.is_stationary};",
            "float z = -9999;",
        ]
        return "\n".join(lines) + "\n"


# --------------------------------------------------------------------------------------
# Synthetic environment
# --------------------------------------------------------------------------------------

@dataclasses.dataclass
class FieldSpec:
    """How to synthesise one environment (all draws come from ``seed``)."""

    A: float = 0.5                  # gyre amplitude
    sigma0: float = 0.3             # sigma_k = sigma0 / sigma_base**k
    sigma_base: float = 2.0         # 2 -> 0.3/2^k ; sqrt(2) -> 0.3/2^(k/2)
    obstacle_frac: float = 0.05
    scalar: float = 0.0             # constant value of all_s_mat (0 = no scalar field)
    scalar_wave: float = 0.0        # amplitude of a smooth scalar pattern added on top
    seed: int = 0


def _fourier_mode(rng: np.random.Generator, X: np.ndarray, Y: np.ndarray, L: float) -> np.ndarray:
    acc = np.zeros_like(X)
    for _ in range(3):
        kx, ky = rng.integers(1, 4, size=2)
        px, py = rng.uniform(0, 2 * math.pi, size=2)
        amp = rng.uniform(0.5, 1.0)
        acc += amp * np.cos(2 * math.pi * kx * X / L + px) * np.cos(2 * math.pi * ky * Y / L + py)
    m = np.max(np.abs(acc))
    return acc / (m if m > 0 else 1.0)


def field_parts(prob: Problem, spec: FieldSpec) -> Dict[str, np.ndarray]:
    """The time-invariant pieces of the seeded fields: u2, v2, s2 (g, g),
    ui1, vi1 (nm, g, g), obs (g, g), and Yi (nt, nrzns, nm).  ``make_fields``
    repeats them over t; a device copy can do the same without host copies."""
    prob.validate()
    g, nt, nm, nr = prob.gsize, prob.nt, prob.nmodes, prob.nrzns
    ss = np.random.SeedSequence(spec.seed)
    r_modes, r_y, r_obs, r_s = [np.random.default_rng(s) for s in ss.spawn(4)]
    xs, ys = prob.grid_ticks()
    X = xs.astype(np.float64)[None, :].repeat(g, 0)             # x varies along j
    Yc = ys.astype(np.float64)[::-1][:, None].repeat(g, 1)      # row i has y = ys[g-1-i]
    L = g * prob.dx
    u2 = -spec.A * np.sin(math.pi * X / L) * np.cos(math.pi * Yc / L)
    v2 = spec.A * np.cos(math.pi * X / L) * np.sin(math.pi * Yc / L)
    ui1 = np.stack([_fourier_mode(r_modes, X, Yc, L) for _ in range(nm)]).astype(np.float32)
    vi1 = np.stack([_fourier_mode(r_modes, X, Yc, L) for _ in range(nm)]).astype(np.float32)
    sig = np.array([spec.sigma0 / (spec.sigma_base ** k) for k in range(nm)], dtype=np.float64)
    Yi = (r_y.standard_normal((nt, nr, nm)) * sig[None, None, :]).astype(np.float32)
    s2 = np.full((g, g), spec.scalar, dtype=np.float64)
    if spec.scalar_wave:
        s2 = s2 + spec.scalar_wave * _fourier_mode(r_s, X, Yc, L)
    obs = (r_obs.random((g, g)) < spec.obstacle_frac).astype(np.int32)
    ts = prob.term_subgrid_size
    obs[prob.i_term:prob.i_term + ts, prob.j_term:prob.j_term + ts] = 0
    return {"u2": u2.astype(np.float32), "v2": v2.astype(np.float32), "ui1": ui1, "vi1": vi1,
            "Yi": Yi, "s2": s2.astype(np.float32), "obs": obs}


def expand_parts(prob: Problem, parts: Dict[str, np.ndarray], broadcast) -> Dict:
    """Repeat the time-invariant parts over t with ``broadcast(array, shape)``."""
    g, nt, nm = prob.gsize, prob.nt, prob.nmodes
    return {"u": broadcast(parts["u2"], (nt, g, g)), "v": broadcast(parts["v2"], (nt, g, g)),
            "ui": broadcast(parts["ui1"], (nt, nm, g, g)), "vi": broadcast(parts["vi1"], (nt, nm, g, g)),
            "Yi": parts["Yi"], "s": broadcast(parts["s2"], (nt, g, g)),
            "mask": broadcast(parts["obs"], (nt, g, g))}


def make_fields(prob: Problem, spec: FieldSpec) -> Dict[str, np.ndarray]:
    """Seeded fields in the reference layout (see the module docstring).

    Mean flow: ``u = -A sin(pi x/L) cos(pi y/L)``, ``v = A cos(pi x/L) sin(pi y/L)``
    with ``L = g*dx`` at cell centres, time invariant.  Modes: per k, an
    independent low-frequency Fourier field for ui and for vi, normalised to
    unit max, time invariant.  Coefficients ``Y[t, rzn, k] ~ N(0, sigma_k)``
    independent over (t, rzn, k).  Obstacles: i.i.d. cells with probability
    ``obstacle_frac``, constant over t, never on the terminal subgrid.
    """
    parts = field_parts(prob, spec)
    return expand_parts(prob, parts, lambda a, shape: np.ascontiguousarray(np.broadcast_to(a, shape)))


def write_reference_inputs(dirpath: str, fields: Dict[str, np.ndarray]) -> None:
    """Write the seven input files with the reference's names and dtypes."""
    os.makedirs(dirpath, exist_ok=True)
    for k, fn in FIELD_FILES.items():
        arr = fields[k]
        want = np.int32 if k == "mask" else np.float32
        np.save(os.path.join(dirpath, fn), np.ascontiguousarray(arr, dtype=want))


def read_reference_inputs(dirpath: str) -> Dict[str, np.ndarray]:
    out = {}
    for k, fn in FIELD_FILES.items():
        out[k] = np.load(os.path.join(dirpath, fn))
    return out


# --------------------------------------------------------------------------------------
# Named workloads
# --------------------------------------------------------------------------------------

def config(name: str, seed: int = 1234) -> Tuple[Problem, FieldSpec]:
    """Named workloads.

    * ``c1`` - 50x50 grid, nt=30, 8 headings, F=1, nrzns=500, 4 modes with
      sigma_k=0.3/2^k, gyre A=0.5, 5% obstacles, target (45, 25).
    * ``c2`` - 200x200 grid, nt=120, 16 headings, F=1, nrzns=5000, 10 modes with
      sigma_k=0.3/2^(k/2), gyre A=1.0, 3% obstacles, target (180, 100).
    * ``c3`` - 300x300 grid, nt=150, 16 headings, nrzns=2000, 8 modes, sigma and
      gyre as c2, 3% obstacles, target (270, 150); counts stored as uint16.
    * small ``t*`` cases for parity tests.
    """
    if name == "c1":
        return (Problem(gsize=50, nt=30, nrzns=500, nmodes=4, num_ac_angles=8, F=1.0,
                        i_term=45, j_term=25, prob_name="synthetic_c1"),
                FieldSpec(A=0.5, sigma0=0.3, sigma_base=2.0, obstacle_frac=0.05, seed=seed))
    if name == "c2":
        return (Problem(gsize=200, nt=120, nrzns=5000, nmodes=10, num_ac_angles=16, F=1.0,
                        i_term=180, j_term=100, prob_name="synthetic_c2"),
                FieldSpec(A=1.0, sigma0=0.3, sigma_base=math.sqrt(2.0), obstacle_frac=0.03, seed=seed))
    if name == "c3":
        return (Problem(gsize=300, nt=150, nrzns=2000, nmodes=8, num_ac_angles=16, F=1.0,
                        i_term=270, j_term=150, prob_name="synthetic_c3"),
                FieldSpec(A=1.0, sigma0=0.3, sigma_base=math.sqrt(2.0), obstacle_frac=0.03, seed=seed))
    if name == "t_time":       # small, obstacles, late penalty active on every layer
        return (Problem(gsize=16, nt=8, nrzns=96, nmodes=3, num_ac_angles=8, F=1.0,
                        i_term=12, j_term=5, neighb_gsize=11, prob_name="t_time"),
                FieldSpec(A=0.6, obstacle_frac=0.08, seed=seed))
    if name == "t_custom":     # two speeds x 8 headings, custom1 reward, 2x2 terminal subgrid
        return (Problem(gsize=20, nt=25, nrzns=130, nmodes=4, num_ac_speeds=2, num_ac_angles=8,
                        F=2.0, i_term=4, j_term=14, term_subgrid_size=2, neighb_gsize=13,
                        prob_type="custom1", alpha=0.05, r_outbound=-1000.0,
                        prob_name="t_custom"),
                FieldSpec(A=0.8, obstacle_frac=0.04, seed=seed))
    if name == "t_energy2":    # radiation reward with a non-zero scalar field, dx != 1
        return (Problem(gsize=18, nt=10, nrzns=70, nmodes=2, num_ac_angles=12, F=1.0,
                        dx=0.5, dy=0.5, dt=0.5, i_term=3, j_term=3, neighb_gsize=15,
                        prob_type="energy2", prob_name="t_energy2"),
                FieldSpec(A=0.4, obstacle_frac=0.05, scalar=0.2, scalar_wave=0.5, seed=seed))
    if name == "t_wide":       # strong noise: samples spread beyond a 7x7 neighbourhood
        return (Problem(gsize=24, nt=6, nrzns=400, nmodes=4, num_ac_angles=8, F=1.0,
                        i_term=20, j_term=20, neighb_gsize=21, prob_name="t_wide"),
                FieldSpec(A=0.5, sigma0=1.2, sigma_base=1.5, obstacle_frac=0.03, seed=seed))
    # The single-large-solve and precision workloads in small: their heading
    # count, mode count, realisation count, gyre and noise, on a small grid.
    if name == "t_m10":        # 200x200x120's per-row shape: 16 headings, 10 modes, 5000 realisations
        return (Problem(gsize=22, nt=4, nrzns=5000, nmodes=10, num_ac_angles=16, F=1.0,
                        i_term=18, j_term=10, neighb_gsize=21, prob_name="t_m10"),
                FieldSpec(A=1.0, sigma0=0.3, sigma_base=math.sqrt(2.0), obstacle_frac=0.03, seed=seed))
    if name == "t_m8":         # 300x300x150's: 16 headings, 8 modes, 2000 realisations
        return (Problem(gsize=27, nt=5, nrzns=2000, nmodes=8, num_ac_angles=16, F=1.0,
                        i_term=24, j_term=13, neighb_gsize=21, prob_name="t_m8"),
                FieldSpec(A=1.0, sigma0=0.3, sigma_base=math.sqrt(2.0), obstacle_frac=0.03, seed=seed))
    if name == "t_m6":         # 6 modes, 2 speeds x 16 headings (32 actions), odd realisation count
        return (Problem(gsize=21, nt=5, nrzns=1537, nmodes=6, num_ac_speeds=2, num_ac_angles=16,
                        F=1.5, i_term=3, j_term=17, neighb_gsize=21, prob_name="t_m6"),
                FieldSpec(A=1.0, sigma0=0.3, sigma_base=math.sqrt(2.0), obstacle_frac=0.04, seed=seed))
    if name == "t_energy1":    # reward type energy1, 5 modes (odd count), 12 headings x 2 speeds
        return (Problem(gsize=17, nt=7, nrzns=300, nmodes=5, num_ac_speeds=2, num_ac_angles=12,
                        F=1.5, i_term=8, j_term=12, term_subgrid_size=2, neighb_gsize=13,
                        prob_type="energy1", prob_name="t_energy1"),
                FieldSpec(A=0.7, obstacle_frac=0.05, seed=seed))
    if name == "t_half":       # time reward with half-cell spacing: remainderf snapping, no scalar field
        return (Problem(gsize=20, nt=7, nrzns=200, nmodes=4, num_ac_angles=16, F=1.0,
                        dx=0.5, dy=0.5, dt=0.5, i_term=6, j_term=15, neighb_gsize=13,
                        prob_name="t_half"),
                FieldSpec(A=0.5, sigma0=0.25, obstacle_frac=0.04, seed=seed))
    if name == "t_energy3":    # reward type energy3 with a scalar field, dx != 1
        return (Problem(gsize=19, nt=9, nrzns=256, nmodes=6, num_ac_angles=8, F=1.0,
                        dx=0.5, dy=0.5, dt=0.5, i_term=14, j_term=4, neighb_gsize=15,
                        prob_type="energy3", prob_name="t_energy3"),
                FieldSpec(A=0.4, obstacle_frac=0.05, scalar=0.3, scalar_wave=0.4, seed=seed))
    raise KeyError(name)
