"""The reference arm of bench.py assembles its JSON line without a GPU when the
reference programs are replaced by a stand-in that returns their timings: every
key the line needs is computed (a name error there would cost the whole arm)."""
import json
import os
import types

import numpy as np

import bench
from oracle import run_ref


def test_reference_arm_line(monkeypatch):
    calls = []

    def fake_run(name, workdir, **kw):
        calls.append(name)
        return {"name": name, "wall_build_s": 40.0, "wall_convert_s": 2.0, "wall_solve_s": 5.0,
                "build_loop_s": 39.0, "solve_total_s": 4.5, "iterations": 120, "final_sup_norm": 0.05,
                "model_dir": workdir}

    monkeypatch.setattr(run_ref, "have_reference", lambda name: True)
    monkeypatch.setattr(run_ref, "run", fake_run)
    args = types.SimpleNamespace(steps=2, warmup=1)
    line = bench.run_reference(args, 1, 0, 0)
    json.dumps(line)
    assert line["impl"] == "reference" and line["metric"] == "build+VI sec"
    assert line["value"] == 47.0 and line["unit"] == "s" and line["higher_is_better"] is False
    assert line["e2e"]["value"] == 47.0 and line["cpu_baseline"]["kind"] == "reference"
    assert calls == ["t_time", bench.WORKLOAD, bench.WORKLOAD]
    assert bench.run_reference(args, 2, 1, 1) is None  # ranks > 0: no work, no line


def test_reference_arm_unavailable(monkeypatch):
    monkeypatch.setattr(run_ref, "have_reference", lambda name: False)
    line = bench.run_reference(types.SimpleNamespace(steps=1, warmup=1), 1, 0, 0)
    assert line["impl"] == "reference" and "unavailable" in line


def test_both_arms_share_the_workload_config(monkeypatch):
    from e2e_gpu_dp_b200.problem import config

    monkeypatch.setattr(run_ref, "have_reference", lambda name: True)
    monkeypatch.setattr(run_ref, "run", lambda name, workdir, **kw: {
        "wall_build_s": 1.0, "wall_convert_s": 0.0, "wall_solve_s": 1.0, "build_loop_s": 1.0,
        "solve_total_s": 1.0, "iterations": 1})
    line = bench.run_reference(types.SimpleNamespace(steps=1, warmup=0), 1, 0, 0)
    prob, _ = config(bench.WORKLOAD)
    assert line["config"] == bench.workload_config(prob, 1)


def test_parity_sample_counts_planted_mismatches():
    """The bench's row-sample comparison: oracle blocks against a whole model
    built by the oracle agree; a count changed in the model copy (planted on
    the CPU) is reported as one mismatched row."""
    import numpy as np

    from oracle import pyoracle as O
    from tests.helpers import problem

    prob, fields = problem("t_time")
    h = O.build_model(prob, fields, nthreads=2)
    h = {"row_ptr": h["row_ptr"], "col": h["col"].astype(np.int32), "cnt": h["cnt"], "R": h["R_full"]}
    blocks = [(r0, O.build_rows(prob, fields, r0=r0, r1=r0 + 300, nthreads=2)) for r0 in (0, 1000, 4000)]
    ok = bench.parity_sample(h, blocks)
    assert ok["rows"] == 900 and ok["mismatched_rows"] == 0 and ok["entries"] > 0
    bad = dict(h)
    bad["cnt"] = h["cnt"].copy()
    k = int(h["row_ptr"][1010])
    bad["cnt"][k] += 1
    assert bench.parity_sample(bad, blocks)["mismatched_rows"] == 1


def test_vi_bytes_and_issue_roofline():
    # per-state row pointer formula: nnz*(b_cnt+4) + (Ns+1)*4 + Na*Ns*4 + 3*Ns*4
    assert bench.vi_bytes_per_iteration(10, 2, 7, 2) == 7 * 6 + 11 * 4 + 2 * 10 * 4 + 3 * 10 * 4
    r = bench.k1_issue_roofline(samples=32 * 10**9, k1_s=1.0, sm_mhz=1000.0, n_sm=100)
    assert r is not None and r["peak"] == 100 * 4 * 1e9
    assert abs(r["achieved"] - r["warp_inst_per_sample"] * 32e9) < 1e-3


def test_assembly_bytes():
    # entries read and written, row offsets read, row pointers written
    assert bench.assembly_bytes(100, 10, 2, 32) == 2 * 100 * 6 + 10 * 4 + 11 * 4
    assert bench.assembly_bytes(100, 10, 4, 64) == 2 * 100 * 8 + 10 * 4 + 11 * 8


def test_parity_sample_counts_each_row_once():
    """A row one entry longer on the device is one mismatched row; the rows
    after it still compare equal."""
    import numpy as np

    from oracle import pyoracle as O
    from tests.helpers import problem

    prob, fields = problem("t_time")
    full = O.build_model(prob, fields, nthreads=2)
    r0 = 1000
    blk = O.build_rows(prob, fields, r0=r0, r1=r0 + 200, nthreads=2)
    rp = full["row_ptr"].copy()
    k = int(rp[r0 + 10])
    col = np.insert(full["col"].astype(np.int32), k, 7)
    cnt = np.insert(full["cnt"], k, 1)
    rp[r0 + 11:] += 1
    h = {"row_ptr": rp, "col": col, "cnt": cnt, "R": full["R_full"]}
    assert bench.parity_sample(h, [(r0, blk)])["mismatched_rows"] == 1


def test_small_case_cpu_leg():
    """The host half of the 50x50 leg: the oracle builds and solves the whole
    workload (a failure there would only show on the GPU box)."""
    cpu, prob, fields, m, V64 = bench.small_case_cpu(threads=max(1, min(8, os.cpu_count() or 1)))
    assert prob.gsize == 50 and prob.nt == 30 and prob.num_actions == 8 and prob.nrzns == 500
    assert cpu["build_s"] > 0 and cpu["solve_s"] > 0
    assert len(m["row_ptr"]) == (prob.nt - 1) * prob.ncells * prob.num_actions + 1
    assert len(V64) == prob.ns and np.all(np.isfinite(V64))
