"""Seeded workload generators for the batched and served forms.

* ``batch_instances`` - many independent planning problems of uneven size:
  grid side uniform in [32, 160], nt in [20, 100], 8 or 16 headings, nrzns in
  [200, 2000], 4-8 modes, a random target cell and start cell, and a 0-5%
  obstacle mask per instance, all drawn from one seed.
* ``serve_fields`` / ``request_stream`` - shared resident fields (one per size
  class drawn from the same distribution, plus large 300x300x150 classes) and
  a Poisson stream of plan requests, each choosing a field, a heading set and
  its own start and target.

Rewards are the reference's "time" type (-dt per step, r_outbound = -100,
r_terminal = +100), so every reward sum is an integer.
"""
import dataclasses
import math
from typing import Dict, List, Tuple

import numpy as np

from .problem import FieldSpec, Problem, expand_parts, field_parts


@dataclasses.dataclass
class Instance:
    prob: Problem
    spec: FieldSpec
    start: Tuple[int, int]


def _draw_problem(rng: np.random.Generator, name: str, g: int, nt: int, na: int, nrzns: int,
                  nm: int) -> Tuple[Problem, Tuple[int, int]]:
    it, jt = (int(x) for x in rng.integers(0, g, size=2))
    si, sj = (int(x) for x in rng.integers(0, g, size=2))
    p = Problem(gsize=g, nt=nt, nrzns=nrzns, nmodes=nm, num_ac_angles=na, F=1.0, i_term=it,
                j_term=jt, neighb_gsize=min(21, g if g % 2 == 1 else g - 1), prob_name=name)
    return p, (si, sj)


def batch_instances(n: int = 256, seed: int = 2024, g_range=(32, 160), nt_range=(20, 100),
                    nrzns_range=(200, 2000), modes_range=(4, 8), obstacle_max=0.05) -> List[Instance]:
    """``n`` problems with the uneven sizes above, all from ``seed``."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        g = int(rng.integers(g_range[0], g_range[1] + 1))
        nt = int(rng.integers(nt_range[0], nt_range[1] + 1))
        na = int(rng.choice([8, 16]))
        nr = int(rng.integers(nrzns_range[0], nrzns_range[1] + 1))
        nm = int(rng.integers(modes_range[0], modes_range[1] + 1))
        p, start = _draw_problem(rng, f"batch_{k}", g, nt, na, nr, nm)
        spec = FieldSpec(A=1.0, sigma0=0.3, sigma_base=math.sqrt(2.0),
                         obstacle_frac=float(rng.uniform(0.0, obstacle_max)), seed=int(rng.integers(1 << 31)))
        out.append(Instance(p, spec, start))
    return out


def device_fields(prob: Problem, spec: FieldSpec, device="cuda") -> Dict:
    """``make_fields`` as CUDA tensors: the time-invariant pieces are built on
    the host and repeated over t on the device (same values)."""
    import torch
    parts = field_parts(prob, spec)

    def bcast(a, shape):
        t = torch.from_numpy(np.ascontiguousarray(a)).to(device)
        return t.expand(*shape).contiguous()

    f = expand_parts(prob, parts, bcast)
    f["Yi"] = torch.from_numpy(parts["Yi"]).to(device)
    return f


@dataclasses.dataclass
class FieldClass:
    fid: int
    prob: Problem      # grid, nt, nrzns, modes (target and headings come with each request)
    spec: FieldSpec


def serve_fields(n_fields: int = 16, n_large: int = 1, seed: int = 77) -> List[FieldClass]:
    """Resident fields: ``n_fields - n_large`` size classes drawn like
    ``batch_instances`` and ``n_large`` 300x300x150 classes (nrzns 2000, 8 modes)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_fields):
        if k >= n_fields - n_large:
            g, nt, nr, nm = 300, 150, 2000, 8
        else:
            g = int(rng.integers(32, 161))
            nt = int(rng.integers(20, 101))
            nr = int(rng.integers(200, 2001))
            nm = int(rng.integers(4, 9))
        p = Problem(gsize=g, nt=nt, nrzns=nr, nmodes=nm, num_ac_angles=16, F=1.0, i_term=0, j_term=0,
                    neighb_gsize=min(21, g if g % 2 == 1 else g - 1), prob_name=f"field_{k}")
        spec = FieldSpec(A=1.0, sigma0=0.3, sigma_base=math.sqrt(2.0),
                         obstacle_frac=float(rng.uniform(0.0, 0.05)), seed=int(rng.integers(1 << 31)))
        out.append(FieldClass(k, p, spec))
    return out


@dataclasses.dataclass
class Request:
    arrival_s: float
    fid: int
    headings: int
    target: Tuple[int, int]
    start: Tuple[int, int]


def request_stream(fields: List[FieldClass], n: int, rate: float, large_frac: float = 0.02,
                   seed: int = 5) -> List[Request]:
    """``n`` requests with exponential inter-arrival times of mean 1/rate; a
    request picks a large field with probability ``large_frac``, else one of
    the other fields uniformly, 8 or 16 headings, and random target and start
    cells (a target on an obstacle cell is still terminal, as in the reference,
    src/build_model.cu:523)."""
    rng = np.random.default_rng(seed)
    small = [f for f in fields if f.prob.gsize < 300]
    large = [f for f in fields if f.prob.gsize >= 300] or small
    t = 0.0
    out = []
    for _ in range(n):
        t += float(rng.exponential(1.0 / rate))
        f = large[int(rng.integers(len(large)))] if rng.random() < large_frac else small[int(rng.integers(len(small)))]
        g = f.prob.gsize
        out.append(Request(t, f.fid, int(rng.choice([8, 16])), (int(rng.integers(g)), int(rng.integers(g))),
                           (int(rng.integers(g)), int(rng.integers(g)))))
    return out


def with_target(prob: Problem, headings: int, target: Tuple[int, int]) -> Problem:
    """The plain per-request problem: the field's grid with this heading set and
    a one-cell terminal subgrid at the target (a served request's terminal)."""
    return dataclasses.replace(prob, num_ac_angles=headings, i_term=int(target[0]), j_term=int(target[1]),
                               term_subgrid_size=1)
