"""Make the golden fixtures of tests/golden/ from runs of the reference itself.

Recipe (the reference's programs need a GPU; its sources are needed only to
compile them):

1. ``python oracle/build_ref.py t_time t_custom t_energy2 t_wide c1``
   compiles the reference's src/build_model.cu and src/spvi_2.cu (unmodified,
   for sm_100a) into oracle/_ref/.
2. On a B200: ``python oracle/run_ref.py t_time t_custom t_energy2 t_wide c1
   --out <dir> --save`` runs build_model -> int64->int32 convert -> spvi_2 on
   the seeded inputs of e2e_gpu_dp_b200.problem.config(name) and saves every
   output array to <dir>/ref_<name>.npz.
3. On the same kind of GPU: ``python tests/golden/make_golden.py --trig
   <dir>`` records the device's cosf/sinf of the action headings (the values
   the reference's move() uses) into <dir>/trig_<name>.npy via the package's
   e2e_action_table.
4. Anywhere: ``python tests/golden/make_golden.py <dir>`` writes the compact
   fixtures tests/golden/ref_<name>.npz.

Compact encoding (lossless): S1 as first differences, S2 relative to the start
of the row's next layer, Val as integer counts (the test checks that
count/nrzns reproduces every stored Val bit for bit), policy/value/R as is, and
a SHA-256 of the regenerated input fields so a change of the input generator
is detected instead of silently compared.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

NAMES = ["t_time", "t_custom", "t_energy2", "t_wide", "c1", "t_m10", "t_m8", "t_m6", "t_energy1", "t_energy3",
         "t_half"]


def fields_digest(fields) -> str:
    h = hashlib.sha256()
    for k in ("u", "v", "ui", "vi", "Yi", "s", "mask"):
        a = np.ascontiguousarray(fields[k])
        h.update(k.encode())
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def encode(prob, ref) -> dict:
    S1 = ref["master_cooS1"].reshape(-1).astype(np.int64)
    S2 = ref["master_cooS2"].reshape(-1).astype(np.int64)
    val = ref["master_cooVal"].reshape(-1).astype(np.float32)
    Ns, nc = prob.ns, prob.ncells
    s_of = S1 % Ns
    next_layer = (s_of // nc + 1) * nc
    cnt = np.rint(val.astype(np.float64) * prob.nrzns).astype(np.int64)
    assert np.all(cnt >= 1) and np.all(cnt <= prob.nrzns)
    assert np.array_equal((cnt.astype(np.float32) / np.float32(prob.nrzns)).astype(np.float32), val)
    return {
        "S1_diff": np.diff(S1, prepend=0).astype(np.int32),
        "S2_rel": (S2 - next_layer).astype(np.int32),
        "count": cnt.astype(np.uint16 if prob.nrzns < 65536 else np.uint32),
        "R": ref["master_R"].reshape(-1).astype(np.float32),
        "policy": ref["policy"].reshape(-1).astype(np.uint32),
        "value": ref["value_function"].reshape(-1).astype(np.float32),
        "prob_params": ref["prob_params"].reshape(-1).astype(np.float32),
        "DP_relv_params": ref["DP_relv_params"].reshape(-1).astype(np.int64),
    }


def decode(prob, fx) -> dict:
    """Inverse of encode(): the reference's arrays exactly as it wrote them."""
    S1 = np.cumsum(fx["S1_diff"].astype(np.int64))
    Ns, nc = prob.ns, prob.ncells
    next_layer = ((S1 % Ns) // nc + 1) * nc
    S2 = fx["S2_rel"].astype(np.int64) + next_layer
    val = (fx["count"].astype(np.float32) / np.float32(prob.nrzns)).astype(np.float32)
    return {"S1": S1, "S2": S2, "val": val, "count": fx["count"].astype(np.int64),
            "R": fx["R"], "policy": fx["policy"], "value": fx["value"],
            "prob_params": fx["prob_params"], "DP_relv_params": fx["DP_relv_params"]}


def record_trig(src: str, names) -> None:
    from e2e_gpu_dp_b200.problem import config
    from e2e_gpu_dp_b200 import api

    for n in names:
        prob, _ = config(n)
        tab = api.action_table(prob)
        np.save(os.path.join(src, f"trig_{n}.npy"), np.stack([tab["cos"], tab["sin"]]))


def main() -> int:
    from e2e_gpu_dp_b200.problem import config, make_fields

    ap = argparse.ArgumentParser()
    ap.add_argument("src")
    ap.add_argument("--trig", action="store_true", help="record device trig values into src")
    ap.add_argument("--names", nargs="*", default=None, help="problems (default: the fixture set)")
    a = ap.parse_args()
    names = a.names or NAMES
    if a.trig:
        record_trig(a.src, names)
        return 0
    for n in names:
        p = os.path.join(a.src, f"ref_{n}.npz")
        if not os.path.exists(p):
            print("missing", p)
            continue
        prob, spec = config(n)
        fields = make_fields(prob, spec)
        fx = encode(prob, np.load(p))
        fx["fields_sha256"] = np.frombuffer(bytes.fromhex(fields_digest(fields)), dtype=np.uint8)
        tp = os.path.join(a.src, f"trig_{n}.npy")
        if os.path.exists(tp):
            fx["device_trig"] = np.load(tp).astype(np.float32)
        out = os.path.join(HERE, f"ref_{n}.npz")
        np.savez_compressed(out, **fx)
        print(n, os.path.getsize(out), "bytes")
    return 0


if __name__ == "__main__":
    sys.exit(main())
