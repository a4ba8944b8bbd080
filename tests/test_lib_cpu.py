"""CPU-side checks of the C-ABI library and the host logic (no GPU calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from e2e_gpu_dp_b200 import _lib
from e2e_gpu_dp_b200.problem import Problem, config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    txt = open(os.path.join(ROOT, "include", "e2e_dp.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(e2e_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _header_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, n
    assert L.e2e_abi_version() == 2


def test_status_strings():
    L = _lib.lib()
    assert L.e2e_status_string(0) == b"ok"
    assert L.e2e_status_string(3) == b"out of memory"


def test_prob_params_round_trip_through_the_library():
    prob, _ = config("t_custom")
    pp = prob.prob_params()
    cp = _lib.Problem()
    L = _lib.lib()
    assert L.e2e_problem_from_params(pp.ctypes.data_as(C.POINTER(C.c_float)), C.byref(cp)) == 0
    assert (cp.gsize, cp.nt, cp.nrzns, cp.num_actions) == (prob.gsize, prob.nt, prob.nrzns, prob.num_actions)
    assert cp.reward_type == 4 and cp.term_subgrid_size == 2
    assert cp.x0 == np.float32(prob.dx) / 2
    out = np.zeros(32, np.float32)
    assert L.e2e_problem_to_params(C.byref(cp), out.ctypes.data_as(C.POINTER(C.c_float))) == 0
    assert np.array_equal(out, pp)


def test_prob_params_slots():
    p = Problem(gsize=50, nt=30, nrzns=500, nmodes=4, num_ac_angles=8, i_term=45, j_term=25)
    pp = p.prob_params()
    assert pp.dtype == np.float32 and pp.shape == (32,)
    assert list(pp[:20]) == [50, 8, 500, 1, 1, -100, 100, 4, 45, 25, 30, 0, 1, 0, 1, 8, 1, 1, 21, 0]
    assert np.all(pp[20:] == -9999)


def test_actions_follow_reference_construction():
    p = Problem(gsize=10, nt=3, nrzns=4, nmodes=1, num_ac_speeds=2, num_ac_angles=4, F=2.0)
    sp, an = p.actions()
    assert list(sp) == [1, 1, 1, 1, 2, 2, 2, 2]
    assert an[1] == np.float32(1 * (2 * np.pi) / 4)
    assert list(an[:4]) == list(an[4:])


def test_header_generation_has_reference_variables():
    prob, _ = config("c1")
    h = prob.reference_header()
    for var in ("prob_type", "prob_name", "alpha_header", "nt", "dt", "gsize", "dx", "dy", "x0",
                "y0", "F", "num_ac_speeds", "num_ac_angles", "num_actions", "nrzns", "bDimx",
                "r_outbound", "r_terminal", "i_term", "j_term", "term_subgrid_size", "nmodes",
                "neighb_gsize", "is_stationary", "z"):
        assert re.search(rf"\b{var}\s*=", h), var


def test_missing_library_fails_loudly(monkeypatch):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", "/nonexistent/libe2edp.so")
    with pytest.raises(ImportError):
        _lib.lib()
