"""Failure paths of the C ABI that need no GPU: malformed model files.

e2e_model_read_npy (the spvi_2 drop-in's get_mdp_model, src/spvi_2.cu:393-504,
which asserts on bad input instead) parses and checks every file before any
device call, so truncated or inconsistent .npy files end with E2E_ERR_IO and
a message, on a machine without a GPU too.
"""
import ctypes as C
import os

import numpy as np
import pytest

from e2e_gpu_dp_b200 import _lib

E2E_ERR_INVALID, E2E_ERR_IO = 1, 4


def _write_model(d, ns=12, na=2):
    rows = np.arange(ns * na, dtype=np.int64)
    S1 = rows.reshape(-1, 1)
    S2 = ((rows % ns + 1) % ns).reshape(-1, 1)
    np.save(os.path.join(d, "master_cooS1.npy"), S1)
    np.save(os.path.join(d, "master_cooS2.npy"), S2)
    np.save(os.path.join(d, "master_cooVal.npy"), np.ones((ns * na, 1), np.float32))
    np.save(os.path.join(d, "master_R.npy"), np.zeros((ns * na, 1), np.float32))
    np.save(os.path.join(d, "DP_relv_params.npy"), np.array([[ns], [na]], np.int64))


def _read(d):
    h = C.c_void_p()
    st = _lib.lib().e2e_model_read_npy(d.encode(), C.byref(h), None)
    msg = _lib.lib().e2e_last_error().decode() if st else ""
    return st, msg


def test_truncated_file_is_an_io_error(tmp_path):
    d = str(tmp_path)
    _write_model(d)
    p = os.path.join(d, "master_cooS2.npy")
    raw = open(p, "rb").read()
    open(p, "wb").write(raw[: len(raw) - 9])
    st, msg = _read(d)
    assert st == E2E_ERR_IO and msg


def test_bad_header_is_an_io_error(tmp_path):
    d = str(tmp_path)
    _write_model(d)
    open(os.path.join(d, "master_R.npy"), "wb").write(b"\x93NUMPY\x01\x00garbage")
    assert _read(d)[0] == E2E_ERR_IO


def test_missing_file_is_an_io_error(tmp_path):
    d = str(tmp_path)
    _write_model(d)
    os.remove(os.path.join(d, "master_cooVal.npy"))
    assert _read(d)[0] == E2E_ERR_IO


@pytest.mark.parametrize("what", ["length", "range", "dtype"])
def test_inconsistent_files_are_io_errors(tmp_path, what):
    d = str(tmp_path)
    _write_model(d)
    if what == "length":
        np.save(os.path.join(d, "master_cooS2.npy"), np.zeros((5, 1), np.int64))
    elif what == "range":
        np.save(os.path.join(d, "master_cooS2.npy"), np.full((24, 1), 99, np.int64))
    else:
        np.save(os.path.join(d, "master_R.npy"), np.zeros((24, 1), np.float64))
    assert _read(d)[0] == E2E_ERR_IO


def test_null_arguments_are_invalid():
    h = C.c_void_p()
    assert _lib.lib().e2e_model_read_npy(None, C.byref(h), None) == E2E_ERR_INVALID
