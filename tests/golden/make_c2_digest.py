"""Make tests/golden/ref_c2_digest.npz: what pins the 200x200x120 workload to
the reference's own output.

The workload's model is too large to commit (2.6e8 entries), so the fixture
keeps the SHA-256 of each model file the reference writes (after the int64 ->
int32 rewrite of src/convert_model_datatype.py:19-23: master_cooS1/S2 int32,
master_cooVal and master_R float32, as (n, 1) arrays), its prob_params and
DP_relv_params, the reference solver's value function and policy at 20000
seeded states, and the digest of the seeded inputs it ran on.

Recipe (the reference's programs need a GPU):

1. ``python oracle/build_ref.py c2`` compiles the reference's
   src/build_model.cu (with the workload's config header) and src/spvi_2.cu,
   unmodified, for sm_100a into oracle/_ref/.
2. On a B200: ``python tests/golden/make_c2_digest.py --out <dir>`` runs
   build_model -> convert -> spvi_2 on problem.config("c2", seed=1234) (about
   a minute) and writes <dir>/ref_c2_digest.npz; copy it to tests/golden/.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

MODEL_FILES = ("master_cooS1", "master_cooS2", "master_cooVal", "master_R")
N_SAMPLE = 20000


def array_sha256(a: np.ndarray) -> bytes:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest()


def sample_states(ns: int, n: int = N_SAMPLE, seed: int = 7) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(ns, size=min(n, ns), replace=False)).astype(np.int64)


def main() -> int:
    from e2e_gpu_dp_b200.problem import config, make_fields
    from oracle import run_ref
    from tests.golden.make_golden import fields_digest

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    prob, spec = config("c2", seed=1234)
    fields = make_fields(prob, spec)
    work = tempfile.mkdtemp(prefix="e2e_c2ref_")
    try:
        r = run_ref.run("c2", os.path.join(work, "c2"), prob=prob, fields=fields, keep_model=False)
        fx = {"fields_sha256": np.frombuffer(bytes.fromhex(fields_digest(fields)), np.uint8)}
        for k in MODEL_FILES:
            arr = np.load(os.path.join(r["model_dir"], k + ".npy"))
            fx[k + "_sha256"] = np.frombuffer(array_sha256(arr), np.uint8)
            fx[k + "_dtype_shape"] = np.array([str(arr.dtype), str(arr.shape)])
        fx["prob_params"] = np.load(os.path.join(r["model_dir"], "prob_params.npy")).reshape(-1)
        fx["DP_relv_params"] = np.load(os.path.join(r["model_dir"], "DP_relv_params.npy")).reshape(-1)
        V = np.load(os.path.join(r["solver_dir"], "value_function.npy")).reshape(-1)
        pi = np.load(os.path.join(r["solver_dir"], "policy.npy")).reshape(-1)
        idx = sample_states(prob.ns)
        fx["sample_states"] = idx
        fx["value_sample"] = V[idx].astype(np.float32)
        fx["policy_sample"] = pi[idx].astype(np.uint32)
        fx["value_max_abs"] = np.array([np.max(np.abs(V.astype(np.float64)))])
        fx["iterations"] = np.array([r["iterations"] or -1])
        os.makedirs(a.out, exist_ok=True)
        np.savez_compressed(os.path.join(a.out, "ref_c2_digest.npz"), **fx)
        print(json.dumps({k: v for k, v in r.items() if k not in ("model_dir", "solver_dir")}))
    finally:
        shutil.rmtree(work, ignore_errors=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
