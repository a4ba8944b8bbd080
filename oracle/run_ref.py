"""Run the reference pipeline (oracle/_ref binaries) on seeded synthetic inputs.

ORACLE -- test infrastructure only (parity checker, golden-vector source and
the reference arm of bench.py).

Mirrors ``make all`` of the reference (``src/Makefile:1-24``) minus plotting:

1. ``build_model <ALPHA*100>`` in a scratch directory holding
   ``data_input/<prob_name>/*.npy`` (``src/build_model.cu:926-1238``);
2. the int64 -> int32 rewrite of ``master_cooS1/S2.npy`` that
   ``src/convert_model_datatype.py:19-23`` performs (done here with numpy, the
   same operation, because the reference tree is not present where this runs);
3. ``spvi_2`` (``src/spvi_2.cu:730-796``), which reads
   ``temp_modelOp_dirName.txt`` and writes ``policy.npy``/``value_function.npy``.

Both programs create their output directories with a non-recursive ``mkdir``
(``src/build_model.cu:1384-1391``), so the ``<prob_type>`` level is created
here beforehand.
"""
from __future__ import annotations

import json
import os
import re
import shutil
import subprocess
import sys
import time
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_DIR = os.path.join(HERE, "_ref")
sys.path.insert(0, ROOT)


def have_reference(name: str) -> bool:
    return os.path.isfile(os.path.join(REF_DIR, name, "build_model")) and os.path.isfile(
        os.path.join(REF_DIR, "spvi_2"))


def run(name: str, workdir: str, seed: int = 1234, fields: Optional[Dict[str, np.ndarray]] = None,
        prob=None, keep_model: bool = True, timeout: float = 3600.0) -> Dict:
    """Run build + convert + solve; return timings, parsed prints and output arrays."""
    from e2e_gpu_dp_b200.problem import config, make_fields, write_reference_inputs

    if prob is None:
        prob, spec = config(name, seed)
        if fields is None:
            fields = make_fields(prob, spec)
    if os.path.exists(workdir):
        shutil.rmtree(workdir)
    os.makedirs(workdir)
    write_reference_inputs(os.path.join(workdir, "data_input", prob.prob_name), fields)
    for top in ("data_modelOutput", "data_solverOutput"):
        os.makedirs(os.path.join(workdir, top, prob.prob_type), exist_ok=True)
    alpha_arg = str(int(round(prob.alpha * 100)))
    t0 = time.perf_counter()
    pb = subprocess.run([os.path.join(REF_DIR, name, "build_model"), alpha_arg], cwd=workdir,
                        capture_output=True, text=True, timeout=timeout)
    t1 = time.perf_counter()
    if pb.returncode != 0:
        raise RuntimeError(f"reference build_model failed ({pb.returncode}): {pb.stderr[-2000:]}")
    with open(os.path.join(workdir, "temp_modelOp_dirName.txt")) as fh:
        lines = fh.read().split("\n")
    model_dir = os.path.join(workdir, lines[4])
    for k in ("master_cooS1.npy", "master_cooS2.npy"):
        p = os.path.join(model_dir, k)
        np.save(p, np.load(p).astype(np.int32))
    t2 = time.perf_counter()
    ps = subprocess.run([os.path.join(REF_DIR, "spvi_2")], cwd=workdir, capture_output=True,
                        text=True, timeout=timeout)
    t3 = time.perf_counter()
    if ps.returncode != 0:
        raise RuntimeError(f"reference spvi_2 failed ({ps.returncode}): {ps.stderr[-2000:]}")
    dur_t = [float(x) for x in re.findall(r"duration@t = ([0-9.eE+-]+)sec", pb.stdout)]
    m_tot = re.search(r"total solve time = ([0-9.eE+-]+)", ps.stdout)
    m_it = re.search(r"num_iterations(\d+)", ps.stdout)
    m_stop = re.search(r"Iteration (\d+): ([0-9.eE+-]+) < ", ps.stdout)
    res = {
        "name": name,
        "wall_build_s": t1 - t0,
        "wall_convert_s": t2 - t1,
        "wall_solve_s": t3 - t2,
        "build_loop_s": float(sum(dur_t)),
        "solve_total_s": float(m_tot.group(1)) if m_tot else None,
        "iterations": int(m_it.group(1)) if m_it else None,
        "final_sup_norm": float(m_stop.group(2)) if m_stop else None,
        "model_dir": model_dir,
    }
    sol_dir = os.path.join(workdir, "data_solverOutput", lines[0], lines[1], lines[2])
    if prob.prob_type == "custom1":
        sol_dir = os.path.join(sol_dir, lines[3])
    res["solver_dir"] = sol_dir
    if keep_model:
        arrs = {}
        for k in ("master_cooS1", "master_cooS2", "master_cooVal", "master_R", "DP_relv_params",
                  "prob_params"):
            arrs[k] = np.load(os.path.join(model_dir, k + ".npy"))
        arrs["policy"] = np.load(os.path.join(sol_dir, "policy.npy"))
        arrs["value_function"] = np.load(os.path.join(sol_dir, "value_function.npy"))
        res["arrays"] = arrs
    return res


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("names", nargs="+")
    ap.add_argument("--workroot", default="/tmp/e2e_refrun")
    ap.add_argument("--out", default=None, help="directory for a JSON summary (and npz if --save)")
    ap.add_argument("--save", action="store_true")
    ap.add_argument("--seed", type=int, default=1234)
    a = ap.parse_args()
    summary = []
    for n in a.names:
        r = run(n, os.path.join(a.workroot, n), seed=a.seed, keep_model=a.save)
        arrs = r.pop("arrays", None)
        print(json.dumps(r), flush=True)
        summary.append(r)
        if a.out and arrs is not None:
            os.makedirs(a.out, exist_ok=True)
            np.savez_compressed(os.path.join(a.out, f"ref_{n}.npz"), **arrs)
        shutil.rmtree(os.path.join(a.workroot, n), ignore_errors=True)
    if a.out:
        os.makedirs(a.out, exist_ok=True)
        with open(os.path.join(a.out, "ref_summary.json"), "w") as fh:
            json.dump(summary, fh, indent=1)
