"""The drop-in executables on the reference's file protocol.

bin/build_model reads input_to_build_model.h and data_input/<prob_name>/*.npy,
writes data_modelOutput/... and temp_modelOp_dirName.txt; after the reference's
int64->int32 convert step, bin/spvi_2 writes data_solverOutput/.../policy.npy and
value_function.npy (src/Makefile:1-24).  Compared with the reference's own
outputs (tests/golden).
"""
import os
import subprocess

import numpy as np
import pytest

from e2e_gpu_dp_b200.problem import write_reference_inputs
from oracle import pyoracle as O
from tests.golden.make_golden import decode
from tests.helpers import VALUE_RTOL, golden, policy_ok, problem, q_values_f64, values_close

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "e2e_gpu_dp_b200", "bin")


@pytest.mark.parametrize("name", ["t_time", "t_custom"])
def test_dropin_pipeline_reproduces_reference_files(tmp_path, name):
    prob, fields = problem(name)
    ref = decode(prob, golden(name))
    wd = str(tmp_path)
    with open(os.path.join(wd, "input_to_build_model.h"), "w") as fh:
        fh.write(prob.reference_header())
    write_reference_inputs(os.path.join(wd, "data_input", prob.prob_name), fields)
    alpha = str(int(round(prob.alpha * 100)))
    r = subprocess.run([os.path.join(BIN, "build_model"), alpha], cwd=wd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = open(os.path.join(wd, "temp_modelOp_dirName.txt")).read().split("\n")
    assert lines[:3] == [prob.prob_type, prob.prob_name, prob.prob_specs()]
    mdir = os.path.join(wd, lines[4])
    S1 = np.load(os.path.join(mdir, "master_cooS1.npy"))
    assert S1.dtype == np.int64
    assert np.array_equal(S1.ravel(), ref["S1"])
    assert np.array_equal(np.load(os.path.join(mdir, "master_cooS2.npy")).ravel(), ref["S2"])
    assert np.array_equal(np.load(os.path.join(mdir, "master_cooVal.npy")).ravel(), ref["val"])
    # the reference's convert step (src/convert_model_datatype.py:19-23)
    for k in ("master_cooS1.npy", "master_cooS2.npy"):
        p = os.path.join(mdir, k)
        np.save(p, np.load(p).astype(np.int32))
    r = subprocess.run([os.path.join(BIN, "spvi_2")], cwd=wd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    sdir = os.path.join(wd, "data_solverOutput", lines[0], lines[1], lines[2])
    if prob.prob_type == "custom1":
        sdir = os.path.join(sdir, lines[3])
    pol = np.load(os.path.join(sdir, "policy.npy"))
    val = np.load(os.path.join(sdir, "value_function.npy"))
    assert pol.dtype == np.uint32 and pol.shape == (prob.ns, 1)
    assert val.dtype == np.float32 and val.shape == (prob.ns, 1)
    orc = O.build_model(prob, fields, nthreads=4)
    nrs = (prob.nt - 1) * prob.ncells
    V64, _, _, _ = O.vi_f64(prob.ns, prob.num_actions, nrs, orc["row_ptr"], orc["col"],
                            cnt=orc["cnt"], scale=prob.nrzns, R=orc["R_full"], mode=1)
    rel, _ = values_close(val.ravel(), V64)
    assert rel <= VALUE_RTOL
    rel_ref, _ = values_close(val.ravel(), ref["value"].astype(np.float64))
    assert rel_ref <= VALUE_RTOL
    Q = q_values_f64(prob, orc["row_ptr"], orc["col"], orc["cnt"], orc["R_full"], V64)
    assert len(policy_ok(Q, pol.ravel().astype(np.int64), V64)) == 0
