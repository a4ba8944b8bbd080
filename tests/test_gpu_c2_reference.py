"""The benchmarked 200x200x120 workload against the reference's own output.

tests/golden/ref_c2_digest.npz (made by tests/golden/make_c2_digest.py from a
run of the reference's build_model -> convert -> spvi_2 on the same seeded
inputs) holds the SHA-256 of the reference's model files: the files the
library writes for the same problem must hash the same, i.e. every next state,
count and reward equal bit for bit.  Values are then checked against an FP64
backward induction on the host (the oracle, over the model copied down from
the device): the library's and the reference's values within VALUE_RTOL, and
neither policy choosing an action outside the FP64 tie band.
"""
import hashlib
import os

import numpy as np
import pytest

from e2e_gpu_dp_b200 import api
from oracle import pyoracle as O
from tests.golden.make_golden import fields_digest
from tests.helpers import GOLDEN, TIE_RTOL, VALUE_RTOL, problem

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(GOLDEN, "ref_c2_digest.npz")
NTHREADS = max(1, min(64, os.cpu_count() or 1))


@pytest.mark.skipif(not os.path.exists(FIXTURE), reason="no reference digest fixture")
def test_c2_model_and_values_match_reference(tmp_path):
    fx = np.load(FIXTURE)
    prob, fields = problem("c2")
    assert fields_digest(fields) == bytes(fx["fields_sha256"]).hex()
    model = api.build_model(prob, fields)
    d = str(tmp_path)
    model.write_npy(d, index_bits=32)  # the reference's files after its int32 convert step
    for k in ("master_cooS1", "master_cooS2", "master_cooVal", "master_R"):
        arr = np.load(os.path.join(d, k + ".npy"))
        assert [str(arr.dtype), str(arr.shape)] == list(fx[k + "_dtype_shape"]), k
        assert hashlib.sha256(np.ascontiguousarray(arr).tobytes()).digest() == bytes(fx[k + "_sha256"]), k
        del arr
    assert np.array_equal(np.load(os.path.join(d, "prob_params.npy")).reshape(-1), fx["prob_params"])
    assert np.array_equal(np.load(os.path.join(d, "DP_relv_params.npy")).reshape(-1), fx["DP_relv_params"])

    V, pi, st = model.solve(method="layered")
    assert st["residual"] == 0.0
    h = model.to_host()
    model.free()
    idx = fx["sample_states"]
    ref_pol = fx["policy_sample"].astype(np.int64).astype(np.int32)  # uint32 -1 -> -1
    V64, _, gap = O.vi_f64_layers(prob.ncells, prob.nt, prob.num_actions, h["row_ptr"], h["col"],
                                  h["cnt"], prob.nrzns, h["R"], policy=pi, nthreads=NTHREADS)
    pol = pi.copy()
    pol[idx] = ref_pol  # the reference's actions at the sampled states
    _, _, gap_ref = O.vi_f64_layers(prob.ncells, prob.nt, prob.num_actions, h["row_ptr"], h["col"],
                                    h["cnt"], prob.nrzns, h["R"], policy=pol, nthreads=NTHREADS)
    scale = float(np.max(np.abs(V64)))
    band = TIE_RTOL * max(1.0, scale)
    assert float(np.max(np.abs(V.astype(np.float64) - V64))) / scale <= VALUE_RTOL
    assert float(np.max(np.abs(fx["value_sample"].astype(np.float64) - V64[idx]))) / scale <= VALUE_RTOL
    assert int(np.sum(gap > band)) == 0               # the library's policy, every state
    assert int(np.sum(gap_ref[idx] > band)) == 0      # the reference's policy at the sample
