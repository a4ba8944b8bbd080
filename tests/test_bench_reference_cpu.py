"""The reference arm of bench.py assembles its JSON line without a GPU when the
reference programs are replaced by a stand-in that returns their timings: every
key the line needs is computed (a name error there would cost the whole arm)."""
import json
import types

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
