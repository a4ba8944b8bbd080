"""Benchmark: end-to-end planner (Monte-Carlo build + value iteration) on one B200.

One step = build the transition model of the single-large-solve workload
(200x200 grid, nt=120, 16 headings, 5000 realisations, 10 modes) and solve it
(layered backward sweep + one FP64-residual verification sweep).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  `value` is seconds per solve with the fields
already resident in HBM; `e2e` is the same through the C ABI from pinned host
buffers (fields host->device and value/policy device->host inside the timed
region).  Extra keys: the fused VI sweep's bandwidth, the dominant kernel's
roofline, the CPU baseline (the oracle port on the host cores) and clocks.
The reference arm runs the reference's own build_model -> convert -> spvi_2
(compiled from its sources into oracle/_ref) on the same workload.
Multi-GPU: independent replicas, one per rank (the workload does not shard).
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import resource
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "c2"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def _peaks():
    try:
        with open(PEAKS_FILE) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class Clocks:
    """SM clock and clock-event-reason samples over the timed region.

    NVML in this process, initialised before the region starts.  Samples are
    taken at step boundaries (``tick``, right after each step's last
    synchronisation, clocks still at their load level) and never while a
    kernel runs: NVML queries issued during the builder's long launches (a
    sampler thread, or nvidia-smi started inside the region) blocked the
    host's CUDA calls and added 0.2-0.7 s to some steps.  nvidia-smi at a
    200 ms period when NVML is absent."""

    # clock event reason bits of NVML (nvmlClocksEventReason*)
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40}
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.samples = []
        self.proc = None
        self.path = None
        self.thread = None

    def _uuid(self):
        import torch

        uuid = str(torch.cuda.get_device_properties(self.dev).uuid)
        return uuid if uuid.startswith("GPU-") else "GPU-" + uuid

    def _sample(self, nv, h):
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        try:
            reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except AttributeError:
            reasons = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        self.samples.append((float(sm), float(smax), int(reasons)))

    def __enter__(self):
        """NVML set-up (before the warm-up steps); sampling starts at begin()."""
        try:
            import pynvml as nv

            nv.nvmlInit()
            try:
                h = nv.nvmlDeviceGetHandleByUUID(self._uuid())
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(self.dev)
            self._sample(nv, h)      # first query outside the timed region
            self.samples.clear()
            self._nv, self._h = nv, h
            self.thread = True       # NVML mode
        except Exception:
            self.thread = None
        return self

    def begin(self):
        """Start of the timed region: NVML samples are taken by tick(); without
        NVML an nvidia-smi sampler runs until exit."""
        if self.thread is not None:
            self.samples.clear()
            return
        try:
            sel = ["-i", self._uuid()]
        except Exception:
            sel = ["-i", str(self.dev)]
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", *sel, f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            t0 = time.time()
            while time.time() - t0 < 10 and os.path.getsize(self.path) == 0:
                time.sleep(0.05)   # its first sample is taken before timing starts
        except Exception:
            self.proc = None

    def tick(self):
        """One sample (NVML mode), called between steps."""
        if self.thread is not None:
            try:
                self._sample(self._nv, self._h)
            except Exception:
                pass

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], [], set()
        if self.thread is not None:
            for a, b, r in self.samples:
                sm.append(a)
                smax.append(b)
                for n, bit in self.REASONS.items():
                    if r & bit:
                        reasons.add(n)
        elif self.path and os.path.exists(self.path):
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            with open(self.path) as fh:
                for line in fh:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        sm.append(float(parts[1]))
                        smax.append(float(parts[2]))
                    except ValueError:
                        continue
                    for n, v in zip(names, parts[5:9]):
                        if v.lower().startswith("active"):
                            reasons.add(n)
            os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax),
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self.thread is not None else "nvidia-smi"}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _max_over_ranks(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_seconds_per_solve(ms_per_step_max: float, ws: int) -> float:
    """Replicas: every rank solves one problem per step, so the job finishes ws
    solves per (slowest rank's) step time."""
    return ms_per_step_max / 1e3 / ws


def _barrier(ws):
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()


def algorithmic_build_bytes(prob, nnz: int, count_bytes: int) -> int:
    """Bytes the builder must move once: fields read once per layer (u, v, the
    2*nmodes mode fields and the mask at t and t+1 per cell, the layer's Y
    coefficients) and the model written (staged CSR entries, per-row offset and R)."""
    nc, nt, nm = prob.ncells, prob.nt, prob.nmodes
    layers = nt - 1
    reads = layers * (nc * (2 + 2 * nm) * 4 + nc * 2 * 4 + prob.nrzns * nm * 4)
    rows = layers * nc * prob.num_actions
    writes = nnz * (4 + count_bytes) + rows * (4 + 4)
    return int(reads + writes)


def workload_config(prob, ws: int = 1) -> dict:
    """The bench line's ``config``: the same dict in both arms."""
    return {
        "workload": "single large solve: 200x200 grid, nt=120, 16 headings, F=1, nrzns=5000, "
                    "10 modes sigma_k=0.3/2^(k/2), gyre A=1, 3% obstacles, seed 1234",
        "states": prob.ns, "rows": (prob.nt - 1) * prob.ncells * prob.num_actions,
        "samples": (prob.nt - 1) * prob.ncells * prob.num_actions * prob.nrzns,
        "parallelism": f"replicas x{ws}", "l2": "inputs (fields 0.45 GB, model 2.2 GB) exceed L2",
    }


def assembly_bytes(nnz: int, n_rows: int, count_bytes: int, index_bits: int) -> int:
    """Bytes the CSR assembly (K2 scan of the tile lengths, K3 copy) must move:
    the staged entries read and the canonical entries written (nnz*(4 +
    b_cnt) each way), the per-row offsets read and the row pointers written
    (4 or 8 bytes)."""
    ptr = 8 if index_bits == 64 else 4
    return int(2 * nnz * (4 + count_bytes) + n_rows * 4 + (n_rows + 1) * ptr)


def vi_bytes_per_iteration(ns: int, na: int, nnz: int, count_bytes: int) -> int:
    """Algorithmic bytes of one VI sweep over the CSR with a per-state row
    pointer: nnz*(b_cnt + 4) + (Ns + 1)*4 + Na*Ns*4 + 3*Ns*4 (entries, row
    pointer, R, V gathered once, V' and the policy written)."""
    return int(nnz * (count_bytes + 4) + (ns + 1) * 4 + na * ns * 4 + 3 * ns * 4)


def k1_issue_roofline(samples: int, k1_s: float, sm_mhz: float, n_sm: int):
    """K1 is bound by instruction issue: warp instructions it issues (per-sample
    count from the ncu capture in profiles/, times the samples) over the SMs'
    issue capacity (4 schedulers x 1 warp instruction per cycle per SM at the
    SM clock measured during the timed steps)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        per_sample = float(json.load(open(path))[f"k_build_tiles/{WORKLOAD}/warp_inst_per_sample"])
    except Exception:
        return None
    inst = per_sample * samples
    achieved = inst / k1_s
    peak = n_sm * 4 * sm_mhz * 1e6
    return {"warp_inst_per_sample": per_sample, "warp_inst": inst, "achieved": achieved, "peak": peak}


def cpu_baseline(prob, fields, threads: int, target_s: float = 15.0, trig=None):
    """The oracle (C restatement) on a bounded sample of rows, extrapolated.
    Returns the baseline and the sampled row blocks [(r0, rows)] (built with
    ``trig``, the device's cos/sin of the headings, so they can be compared
    with the device's rows bit for bit)."""
    from oracle import pyoracle as O

    n_rows = (prob.nt - 1) * prob.ncells * prob.num_actions
    # calibrate on a small block, then run a block sized for ~target_s
    probe = 2048
    t0 = time.perf_counter()
    O.build_rows(prob, fields, trig=trig, r0=n_rows // 2, r1=n_rows // 2 + probe, nthreads=threads)
    dt = time.perf_counter() - t0
    rows = int(min(n_rows, max(probe, probe * target_s / max(dt, 1e-6))))
    chunks = 8
    per = max(1, rows // chunks)
    t0 = time.perf_counter()
    done = 0
    nnz = 0
    blocks = []
    for c in range(chunks):
        r0 = int((c + 0.5) * n_rows / chunks) - per // 2
        out = O.build_rows(prob, fields, trig=trig, r0=r0, r1=r0 + per, nthreads=threads)
        done += per
        nnz += len(out["col"])
        blocks.append((r0, out))
    el = time.perf_counter() - t0
    est_build = el * n_rows / done
    # FP64 backward sweep: time on the sampled rows and scale by nnz
    rp = out["row_ptr"]
    t1 = time.perf_counter()
    for _ in range(3):
        acc = np.add.reduceat(out["cnt"].astype(np.float64) * 1e-3, rp[:-1][np.diff(rp) > 0])
    vi_per_nnz = (time.perf_counter() - t1) / 3 / max(1, len(out["col"]))
    est_nnz = nnz * n_rows / done
    est_vi = vi_per_nnz * est_nnz
    return {
        "value": est_build + est_vi, "unit": "s", "cores": threads, "kind": "port",
        "sample": f"oracle build of {done} of {n_rows} rows ({chunks} blocks spread over the layers) "
                  f"in {el:.1f}s on {threads} threads, extrapolated linearly; VI one FP64 sweep "
                  f"estimated from the sampled rows",
    }, blocks


def parity_sample(h, blocks, integer_rewards: bool = True) -> dict:
    """Device rows against the oracle's rows of the same blocks: each row's
    length, next states and counts bit for bit, rewards bit for bit (integer
    rewards).  Rows are compared one by one (a differing row does not shift
    the comparison of the rows after it)."""
    rows = entries = bad_rows = 0
    for r0, o in blocks:
        n = len(o["row_ptr"]) - 1
        rp = h["row_ptr"][r0:r0 + n + 1].astype(np.int64)
        orp = o["row_ptr"].astype(np.int64)
        glen, olen = np.diff(rp), np.diff(orp)
        bad = glen != olen
        same = np.nonzero(~bad)[0]
        if len(same):
            # entries of the rows of equal length, side by side
            ln = glen[same]
            g_idx = np.repeat(rp[:-1][same], ln) + _ranges(ln)
            o_idx = np.repeat(orp[:-1][same] - orp[0], ln) + _ranges(ln)
            diff = (h["col"][g_idx].astype(np.int64) != o["col"][o_idx].astype(np.int64)) | \
                   (h["cnt"][g_idx].astype(np.int64) != o["cnt"][o_idx].astype(np.int64))
            if diff.any():
                bad[same[np.repeat(np.arange(len(same)), ln)[diff]]] = True
        if integer_rewards:
            bad |= h["R"][r0:r0 + n] != o["R"]
        bad_rows += int(np.sum(bad))
        rows += n
        entries += len(o["col"])
    return {"rows": rows, "entries": entries, "mismatched_rows": bad_rows}


def _ranges(lengths):
    """0..l-1 for every l in lengths, concatenated."""
    lengths = np.asarray(lengths, np.int64)
    if len(lengths) == 0:
        return np.zeros(0, np.int64)
    tot = int(lengths.sum())
    starts = np.repeat(np.cumsum(lengths) - lengths, lengths)
    return np.arange(tot, dtype=np.int64) - starts


def run_ours(args, ws, rank, local):
    import torch

    from e2e_gpu_dp_b200 import api
    from e2e_gpu_dp_b200.problem import config, make_fields

    torch.cuda.set_device(local)
    prob, spec = config(WORKLOAD, seed=1234 + rank)
    fields = make_fields(prob, spec)
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in fields.items()}
    stream = torch.cuda.current_stream()
    V = torch.empty(prob.ns, dtype=torch.float32, device="cuda")
    pi = torch.empty(prob.ns, dtype=torch.int32, device="cuda")

    def step(ev0=None, ev1=None):
        """Build + layered solve between the events ev0/ev1 (both calls return
        after their stream work is done); the model's info and its free come
        after ev1, outside the timed region.  Returns (info, solve stats, host
        ms of the two calls) when timed."""
        if ev0 is not None:
            ev0.record(stream)
        t0 = time.perf_counter()
        m = api.build_model(prob, dev, stream=stream)
        t1 = time.perf_counter()
        _, _, st = m.solve(method="layered", value=V, policy=pi, stream=stream)
        t2 = time.perf_counter()
        if ev1 is None:
            m.free()
            return None
        ev1.record(stream)
        inf = m.info()
        m.free()
        return inf, st, (round((t1 - t0) * 1e3, 1), round((t2 - t1) * 1e3, 1))

    recs = []
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    # the Python collector's pauses are host noise between launches: collect and
    # freeze the objects made so far, and keep it off while steps are timed
    gc.collect()
    gc.freeze()
    with Clocks(local) as clk:
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        _barrier(ws)
        clk.begin()
        gc.collect()
        gc.disable()
        torch.cuda.synchronize()
        # each step between its own events: the clock sample taken between two
        # steps (host only, GPU idle) is not part of either
        for k in range(args.steps):
            r0 = resource.getrusage(resource.RUSAGE_SELF)
            inf, st, host_ms = step(starts[k], ends[k])
            torch.cuda.synchronize()
            r1 = resource.getrusage(resource.RUSAGE_SELF)
            usage = {"cpu_ms": round((r1.ru_utime + r1.ru_stime - r0.ru_utime - r0.ru_stime) * 1e3, 1),
                     "involuntary_switches": r1.ru_nivcsw - r0.ru_nivcsw,
                     "page_faults": r1.ru_minflt - r0.ru_minflt + r1.ru_majflt - r0.ru_majflt}
            recs.append((inf, st, host_ms, usage))
            clk.tick()
        torch.cuda.synchronize()
        gc.enable()
    _barrier(ws)
    step_ms = [round(starts[k].elapsed_time(ends[k]), 2) for k in range(args.steps)]
    ms = _max_over_ranks(sum(starts[k].elapsed_time(ends[k]) for k in range(args.steps)) / args.steps, ws)
    clocks = clk.summary()

    info = recs[-1][0]
    k1_ms = statistics.mean(r[0]["build_kernel_ms"] for r in recs)
    asm_ms = statistics.mean(r[0]["assemble_ms"] for r in recs)
    solve_ms = statistics.mean(r[1]["seconds"] * 1e3 for r in recs)
    pack_ms = statistics.mean(r[1]["pack_ms"] for r in recs)
    pass_ms = statistics.mean(r[1]["sweep_seconds"] * 1e3 for r in recs)
    # trig, build, 3 scan kernels, assemble; pack count, 3 scan kernels, pack fill;
    # the persistent layered sweep and the verification sweep
    launches = 6 + 5 + 2

    # e2e through the C ABI from pinned host memory
    pinned = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory() for k, v in fields.items()}
    hV = torch.empty(prob.ns, dtype=torch.float32).pin_memory()
    hpi = torch.empty(prob.ns, dtype=torch.int32).pin_memory()
    host_fields = {k: t.numpy() for k, t in pinned.items()}
    h2d = int(sum(t.numel() * t.element_size() for t in pinned.values()))
    d2h = int(hV.numel() * 4 + hpi.numel() * 4)

    e2e_split = []

    def e2e_step(record=False):
        t0 = time.perf_counter()
        m = api.build_model(prob, host_fields, stream=stream)
        t1 = time.perf_counter()
        m.solve(method="layered", value=hV, policy=hpi, stream=stream)
        t2 = time.perf_counter()
        m.free()
        if record:
            e2e_split.append((round((t1 - t0) * 1e3, 1), round((t2 - t1) * 1e3, 1)))

    for _ in range(max(1, min(args.warmup, 2))):
        e2e_step()
    torch.cuda.synchronize()
    _barrier(ws)
    gc.collect()
    gc.disable()
    t0 = time.perf_counter()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    e2e_steps = []
    for _ in range(args.steps):
        te = time.perf_counter()
        e2e_step(record=True)
        e2e_steps.append(round((time.perf_counter() - te) * 1e3, 1))
    f1.record(stream)
    torch.cuda.synchronize()
    gc.enable()
    e2e_ms = max(f0.elapsed_time(f1), (time.perf_counter() - t0) * 1e3) / args.steps
    e2e_ms = _max_over_ranks(e2e_ms, ws)

    # the fused VI kernel in the reference's Jacobi schedule (VI SpMV GB/s)
    m = api.build_model(prob, dev, stream=stream)
    _, _, jst = m.solve(method="jacobi", threshold=0.1, value=V, policy=pi, stream=stream)
    _, _, lst = m.solve(method="layered", fp64_check=True, value=V, policy=pi, stream=stream)
    minf = m.info()
    # parity: the device's rows against the oracle's rows of the CPU baseline's
    # sample (same seeded inputs, the device's heading cos/sin), and the values
    # against an FP64 backward induction on the host over the device's model
    check = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        tab = api.action_table(prob)
        baseline, blocks = cpu_baseline(prob, fields, threads=os.cpu_count() or 1,
                                        trig=(tab["cos"], tab["sin"]))
        h = m.to_host()
        check = {"parity_sample": parity_sample(h, blocks)}
        del blocks
        from oracle import pyoracle as O
        Vh = V.cpu().numpy().astype(np.float64)
        pih = pi.cpu().numpy()
        tf = time.perf_counter()
        V64, _, gap = O.vi_f64_layers(prob.ncells, prob.nt, prob.num_actions, h["row_ptr"], h["col"],
                                      h["cnt"], prob.nrzns, h["R"], policy=pih,
                                      nthreads=os.cpu_count() or 1)
        scale = float(np.max(np.abs(V64)))
        band = 2e-5 * max(1.0, scale)
        check["fp64_oracle"] = {
            "kind": "oracle/e2e_oracle.c FP64 backward induction on the host over the device's model",
            "seconds": round(time.perf_counter() - tf, 2),
            "max_rel_err": float(np.max(np.abs(Vh - V64)) / scale),
            "policy_mismatches_outside_ties": int(np.sum(gap > band)),
            "policy_differs_within_ties": int(np.sum((gap > 0) & (gap <= band))),
            "tie_band": band}
        del h, V64, gap
    m.free()
    hbm, peak_kind = _peaks()
    cb = 2 if minf["count_type"] == 0 else 4
    vi_bytes = vi_bytes_per_iteration(prob.ns, prob.num_actions, minf["nnz"], cb)
    vi_gbs = jst["stream_bytes_per_sweep"] * jst["iterations"] / jst["seconds"] / 1e9
    vi_alg_gbs = vi_bytes * jst["iterations"] / jst["seconds"] / 1e9

    # policy rollout evaluation of the solved c2 policy from the reference
    # script's start cell (int(0.5 g), int(0.95 g)), every realisation, against
    # the Python restatement of the reference's trajectory loop on a sample
    start = (int(0.5 * prob.gsize), int(0.95 * prob.gsize))
    m = api.build_model(prob, dev, stream=stream)
    m.solve(method="layered", value=V, policy=pi, stream=stream)
    m.free()
    ro = api.rollout(prob, dev, pi, start, stream=stream)
    ro2 = api.rollout(prob, dev, pi, start, stream=stream)
    ri = api.rollout(prob, dev, pi, start, stream=stream, interpolate=True)
    rollout = {"start": list(start), "realisations": prob.nrzns, "success_rate": ro2["stats"]["success_rate"],
               "mean_time": ro2["stats"]["mean_time"], "kernel_s": round(ro2["stats"]["seconds"], 6),
               "interpolated": {"success_rate": ri["stats"]["success_rate"], "mean_time": ri["stats"]["mean_time"],
                                "kernel_s": round(ri["stats"]["seconds"], 6)}}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import rollout as RO
        pih = pi.cpu().numpy().astype(np.int64)
        n_cpu = 100
        tc = time.perf_counter()
        o = RO.rollout(prob, fields, pih, start, n_rzns=n_cpu, dot="numpy")
        cpu_s = (time.perf_counter() - tc) / n_cpu * prob.nrzns
        same = float(np.mean(o["success"] == ro2["success"][:n_cpu]))
        rollout.update({"cpu_reference_loop_s_extrapolated": round(cpu_s, 3), "cpu_sample": n_cpu,
                        "outcome_agreement_on_sample": same,
                        "speedup_vs_cpu": round(cpu_s / max(ro2["stats"]["seconds"], 1e-9), 1)})

    # fused build+backup (e2e_build_solve): each layer backed up as it is built,
    # no model stored; compared with the build + layered solve just above
    Vf = torch.empty_like(V)
    pif = torch.empty_like(pi)
    api.build_solve(prob, dev, value=Vf, policy=pif, stream=stream)
    fused_ms = []
    for _ in range(3):
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        _, _, fst = api.build_solve(prob, dev, value=Vf, policy=pif, stream=stream)
        g1.record(stream)
        torch.cuda.synchronize()
        fused_ms.append(g0.elapsed_time(g1))
    fused = {"api": "e2e_build_solve", "ms": [round(x, 2) for x in fused_ms],
             "kernel_ms": round(fst["seconds"] * 1e3, 2), "launches": fst["launches"], "nnz": fst["nnz"],
             "identical_to_build_then_solve": bool(torch.equal(Vf, V) and torch.equal(pif, pi)),
             "speedup_vs_step": round(ms / statistics.median(fused_ms), 3)}

    k1_bytes = algorithmic_build_bytes(prob, info["nnz"], cb)
    k1_gbs = k1_bytes / (k1_ms * 1e-3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(f"k_build_tiles/{WORKLOAD}/dram_bytes")
        except Exception:
            traffic = None
    samples = (prob.nt - 1) * prob.ncells * prob.num_actions * prob.nrzns

    value_s = whole_job_seconds_per_solve(ms, ws)
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    sm_mhz = clocks["sm_mhz"] if clocks else 1965.0
    issue = k1_issue_roofline(samples, k1_ms * 1e-3, sm_mhz, n_sm)
    hbm_part = {"achieved": round(k1_gbs, 2), "peak": hbm, "unit": "GB/s", "frac": round(k1_gbs / hbm, 5),
                "traffic": traffic, "peak_source": f"{peak_kind} hbm_gbs", "algorithmic_bytes": k1_bytes}
    if issue is not None:
        roof = {"kernel": "k_build_tiles", "bound": "issue", "achieved": round(issue["achieved"], 1),
                "peak": round(issue["peak"], 1), "unit": "warp-inst/s",
                "frac": round(issue["achieved"] / issue["peak"], 4), "traffic": traffic,
                "warp_inst_per_sample": issue["warp_inst_per_sample"], "sm_mhz": sm_mhz, "sms": n_sm,
                "note": "issue-bound Monte-Carlo kernel: warp instructions (per-sample count of the ncu "
                        "capture in profiles/k_build_tiles_c2nt30.md x samples) / K1 time, against 4 warp "
                        "instructions per cycle per SM at the measured SM clock; its HBM figure below",
                "hbm": hbm_part}
    else:
        roof = {"kernel": "k_build_tiles", "bound": "hbm", **hbm_part}
    asm_bytes = assembly_bytes(info["nnz"], info["n_rows"], cb, info["index_bits"])
    asm_gbs = asm_bytes / (asm_ms * 1e-3) / 1e9 if asm_ms > 0 else None
    asm_roof = {"kernels": "k_scan_* (K2) + k_assemble (K3)", "bound": "hbm", "ms": round(asm_ms, 3),
                "algorithmic_bytes": asm_bytes,
                "achieved": round(asm_gbs, 1) if asm_gbs else None, "peak": hbm, "unit": "GB/s",
                "frac": round(asm_gbs / hbm, 4) if asm_gbs else None}
    line = {
        "metric": "build+VI sec",
        "value": round(value_s, 6),
        "unit": "s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 3),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32 values, u16 counts, fp64 residual",
        "data": "synthetic (seeded double gyre + Fourier modes, reference layout)",
        "config": workload_config(prob, ws),
        "nnz": info["nnz"],
        "solve": "layered backward sweep + FP64-residual verification sweep",
        "e2e": {"value": round(e2e_ms / 1e3 / ws, 6), "unit": "s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "step_wall_ms": e2e_steps,
                "step_build_solve_wall_ms": e2e_split},
        "gpu_launches": launches,
        "step_ms": step_ms, "step_host_ms": [r[2] for r in recs],
        # the calling process per step: CPU time, preemptions, page faults
        "step_host_usage": [r[3] for r in recs],
        "step_phases_ms": [{"build_kernel": round(r[0]["build_kernel_ms"], 2), "assemble": round(r[0]["assemble_ms"], 2),
                            "pack": round(r[1]["pack_ms"], 2), "solve": round(r[1]["seconds"] * 1e3, 2)}
                           for r in recs],
        "phases_ms": {"build_kernel": round(k1_ms, 3), "assemble": round(asm_ms, 3),
                      "pack": round(pack_ms, 3), "solve": round(solve_ms, 3),
                      "layered_pass": round(pass_ms, 3)},
        "roofline": roof,
        "assembly": asm_roof,
        "build_samples_per_s": round(samples / (k1_ms * 1e-3), 1),
        "vi": {"kernel": "k_vi_chunks (Jacobi, reference schedule)", "iterations": jst["iterations"],
               "algorithmic_bytes_per_sweep": vi_bytes,
               "moved_bytes_per_sweep": jst["stream_bytes_per_sweep"], "seconds": round(jst["seconds"], 6),
               "achieved_gbs": round(vi_alg_gbs, 1), "peak": hbm, "frac": round(vi_alg_gbs / hbm, 4),
               "moved_gbs": round(vi_gbs, 1), "moved_frac": round(vi_gbs / hbm, 4),
               "note": "algorithmic bytes per sweep: nnz*(b_cnt+4) + (Ns+1)*4 + Na*Ns*4 + 3*Ns*4 "
                       "(entries, per-state row pointer, R, V gathered once, V' and the policy written); "
                       "moved: the sliced copy actually streamed (packed entries, R, padding)",
               "per_row_pointer_bytes_per_sweep": jst["bytes_per_sweep"],
               "layered_seconds": round(lst["seconds"], 6),
               "layered_pass_seconds": round(lst["sweep_seconds"], 6),
               "fp64_max_rel_err": lst["fp64_max_rel_err"]},
        "rollout": rollout,
        "fused_build_solve": fused,
        "clocks": clocks,
    }
    if check is not None:
        line["cpu_baseline"] = baseline
        line.update(check)
    return line


def run_batched(n_models: int = 256, seed: int = 2024) -> dict:
    """Batched form: ``n_models`` uneven planning problems (grid 32-160, nt
    20-100, 8/16 headings, nrzns 200-2000, 4-8 modes, 0-5% obstacles, random
    targets; one seed), built and solved one at a time through the plain API
    (build_model + layered solve + free), and batched: groups of 32 built
    concurrently and each group solved in one persistent launch.  Then the
    solves alone with all models resident: one launch for all of them against
    the plain solve of one model at a time.  Device-resident seeded fields;
    times are CUDA events on the stream (or wall clock where larger)."""
    import torch

    from e2e_gpu_dp_b200 import api
    from e2e_gpu_dp_b200.workloads import batch_instances, device_fields

    insts = batch_instances(n_models, seed=seed)
    stream = torch.cuda.current_stream()
    fields = [device_fields(x.prob, x.spec) for x in insts]
    outs = [(torch.empty(x.prob.ns, dtype=torch.float32, device="cuda"),
             torch.empty(x.prob.ns, dtype=torch.int32, device="cuda")) for x in insts]
    torch.cuda.synchronize()
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731

    # one warm-up problem for both arms (module loading, pool growth)
    m = api.build_model(insts[0].prob, fields[0], stream=stream)
    m.solve(method="layered", value=outs[0][0], policy=outs[0][1], stream=stream)
    m.free()

    # sequential: build, solve, free, one problem at a time
    solve_s = 0.0
    a, b = ev(), ev()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a.record(stream)
    for x, f, (V, pi) in zip(insts, fields, outs):
        m = api.build_model(x.prob, f, stream=stream)
        _, _, st = m.solve(method="layered", value=V, policy=pi, stream=stream)
        solve_s += st["seconds"] + st["pack_ms"] * 1e-3
        m.free()
    b.record(stream)
    torch.cuda.synchronize()
    seq_s = max(a.elapsed_time(b) / 1e3, time.perf_counter() - t0)
    ref = [(V.clone(), pi.clone()) for V, pi in outs]

    # batched, pipelined: groups of 32 built (e2e_build_models, two host
    # workers: a build's host steps overlap the other's kernels, 4 % faster
    # than one), each group solved in one launch, then freed.  One untimed
    # group first, as the sequential arm's warm-up problem: its launch tunes
    # the schedule (e2e_spvi_solve_batch times its candidates on a new batch
    # shape) and pays the batched path's first-call costs (about 0.85 s on a
    # fresh process); the timed groups reuse that schedule instead of
    # re-tuning on every shape they bring
    group, workers = 32, 2
    models = api.build_models([x.prob for x in insts[:group]], fields[:group], workers=workers)
    first = api.solve_batch(models, [o[0] for o in outs[:group]], [o[1] for o in outs[:group]], stream=stream)
    for mm in models:
        mm.free()
    sch = first["groups"] | (first["tune"] << 4) | 0x100
    for V, pi in outs:
        V.fill_(float("nan"))
        pi.fill_(-7)
    a, c = ev(), ev()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a.record(stream)
    b_build = 0.0
    for g0 in range(0, n_models, group):
        tb = time.perf_counter()
        models = api.build_models([x.prob for x in insts[g0:g0 + group]], fields[g0:g0 + group], workers=workers)
        b_build += time.perf_counter() - tb
        api.solve_batch(models, [o[0] for o in outs[g0:g0 + group]], [o[1] for o in outs[g0:g0 + group]],
                        schedule=sch, stream=stream)
        for mm in models:
            mm.free()
    c.record(stream)
    torch.cuda.synchronize()
    total_s = max(a.elapsed_time(c) / 1e3, time.perf_counter() - t0)
    same = all(torch.equal(V, r[0]) and torch.equal(pi, r[1]) for (V, pi), r in zip(outs, ref))

    # solves alone, all models resident (built untimed): one batched launch
    # (graph replay, tuned schedule) vs the plain API one model at a time
    models = api.build_models([x.prob for x in insts], fields, workers=4)
    api.solve_batch(models, [o[0] for o in outs], [o[1] for o in outs], stream=stream)
    reps = []
    for _ in range(5):
        st2 = api.solve_batch(models, [o[0] for o in outs], [o[1] for o in outs], stream=stream)
        reps.append(st2["seconds"])
    same = same and all(torch.equal(V, r[0]) and torch.equal(pi, r[1]) for (V, pi), r in zip(outs, ref))
    seq_solve_only = []
    a, b = ev(), ev()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a.record(stream)
    for mm, (V, pi) in zip(models, outs):
        _, _, st = mm.solve(method="layered", value=V, policy=pi, stream=stream)
        seq_solve_only.append(st["sweep_seconds"])
    b.record(stream)
    torch.cuda.synchronize()
    seq_resident_s = max(a.elapsed_time(b) / 1e3, time.perf_counter() - t0)
    for mm in models:
        mm.free()
    rows = sum((x.prob.nt - 1) * x.prob.ncells * x.prob.num_actions for x in insts)
    batch_solve_s = statistics.median(reps)
    return {
        "workload": f"{n_models} uneven MDPs: grid 32-160, nt 20-100, 8/16 headings, nrzns 200-2000, "
                    "4-8 modes, 0-5% obstacles, random start/target, seed " + str(seed),
        "models": n_models, "states": int(sum(x.prob.ns for x in insts)), "rows": int(rows),
        "sequential_s": round(seq_s, 4), "sequential_solves_s": round(solve_s, 5),
        "batched_total_s": round(total_s, 4), "batched_build_wall_s": round(b_build, 4),
        "batched_group": group, "build_workers": workers,
        "warmup_group_tune_ms": round(first["tune_ms"], 2),
        "batched_solve_s": round(batch_solve_s, 6),
        "sequential_resident_solves_s": round(seq_resident_s, 5),
        "sequential_layered_passes_s": round(sum(seq_solve_only), 6),
        "solves_per_s_batched": round(n_models / batch_solve_s, 1),
        "solves_per_s_sequential": round(n_models / seq_resident_s, 1),
        "solve_speedup_vs_sequential": round(seq_resident_s / batch_solve_s, 2),
        "total_speedup_vs_sequential": round(seq_s / total_s, 3),
        "schedule": {"warps_per_chunk": st2["groups"], "tune": st2["tune"], "ctas": st2["grid"],
                     "graph": st2["graph"]},
        "sweep_gbs": round(st2["stream_bytes"] / batch_solve_s / 1e9, 1),
        "identical_to_sequential": bool(same),
    }


def run_served(rates=(50, 100, 200, 500, 1000, 2000), seconds_per_rate=10.0, max_requests=20000,
               plain_sample=40) -> dict:
    """Served form: 16 resident fields (15 size classes drawn like the batched
    form plus one 300x300x150 class), Poisson request streams (each request picks
    a field, 8 or 16 headings, a target and a start; 2% pick the large field)
    at each rate for ``seconds_per_rate`` (at most ``max_requests``), through the
    request server; then a burst of requests submitted at once (capacity).  The
    plain path - build the model with the request's target, solve, free - is
    timed one request at a time on a sample of the same stream, and the served
    values at the start cells are compared with it."""
    import threading

    import torch

    from e2e_gpu_dp_b200 import api
    from e2e_gpu_dp_b200.workloads import Request, device_fields, request_stream, serve_fields, with_target

    fcs = serve_fields(16, n_large=1)
    dev = [device_fields(fc.prob, fc.spec) for fc in fcs]
    srv = api.Server(max_batch=256)
    fids = [srv.add_field(fc.prob, f) for fc, f in zip(fcs, dev)]
    assert fids == list(range(len(fcs)))

    large_fids = {fc.fid for fc in fcs if fc.prob.gsize >= 300}

    def serve(reqs, paced=True, srv=srv):
        lat, qd, bs = [], [], []
        lat_small, lat_large = [], []
        results = {}

        def submitter():
            t0 = time.perf_counter()
            for k, r in enumerate(reqs):
                if paced:
                    dt = t0 + r.arrival_s - time.perf_counter()
                    if dt > 0:
                        time.sleep(dt)
                srv.submit(r.fid, r.headings, r.target, r.start, tag=k)
        th = threading.Thread(target=submitter)
        t0 = time.perf_counter()
        th.start()
        while len(results) < len(reqs):
            for res in srv.poll(4096, wait_s=0.05):
                results[res["tag"]] = res
        t1 = time.perf_counter()
        th.join()
        for k, res in results.items():
            lat.append(res["latency_ms"])
            qd.append(res["queue_ms"])
            bs.append(res["batch_size"])
            (lat_large if reqs[k].fid in large_fids else lat_small).append(res["latency_ms"])
        fails = sum(1 for res in results.values() if res["status"] != 0)

        def pct(x, q):
            return round(float(np.percentile(x, q)), 3) if x else None

        return results, {"requests": len(reqs), "failed": fails, "seconds": round(t1 - t0, 4),
                         "solves_per_s": round(len(reqs) / (t1 - t0), 1),
                         "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99),
                         "small": {"requests": len(lat_small), "p50_ms": pct(lat_small, 50),
                                   "p99_ms": pct(lat_small, 99)},
                         "large_300x300x150": {"requests": len(lat_large), "p50_ms": pct(lat_large, 50),
                                               "p99_ms": pct(lat_large, 99)},
                         "mean_queue_ms": round(float(np.mean(qd)), 3),
                         "mean_batch": round(float(np.mean(bs)), 1), "max_batch": int(np.max(bs))}

    # warm-up: every (field, heading set) base model built once (resident afterwards)
    t0 = time.perf_counter()
    warm = [Request(0.0, fid, h, (1, 1), (0, 0)) for fid in range(len(fcs)) for h in (8, 16)]
    serve(warm, paced=False)
    warm_s = time.perf_counter() - t0

    per_rate = []
    for lam in rates:
        n = int(min(max_requests, lam * seconds_per_rate))
        reqs = request_stream(fcs, n, lam, seed=int(lam))
        _, stats = serve(reqs)
        stats["rate"] = lam
        per_rate.append(stats)
    burst_reqs = request_stream(fcs, 5000, 1e9, seed=99)
    burst_res, burst = serve(burst_reqs, paced=False)


    # plain path on a sample of the burst's requests, one at a time
    sample = burst_reqs[:plain_sample]
    plain_lat, err = [], 0.0
    torch.cuda.synchronize()
    tp0 = time.perf_counter()
    for k, r in enumerate(sample):
        fc = fcs[r.fid]
        ts = time.perf_counter()
        m = api.build_model(with_target(fc.prob, r.headings, r.target), dev[r.fid])
        V, pi, _ = m.solve(method="layered")
        m.free()
        plain_lat.append((time.perf_counter() - ts) * 1e3)
        s0 = r.start[0] * fc.prob.gsize + r.start[1]
        sv = burst_res[k]["value_at_start"]
        err = max(err, abs(float(sv) - float(V[s0])) / max(1.0, abs(float(V[s0]))))
    plain_s = time.perf_counter() - tp0
    st = srv.stats()
    srv.close()
    # the same server design without batching: one request per launch, every
    # base model cached as above (isolates continuous batching from caching)
    one = api.Server(max_batch=1)
    for fc, f in zip(fcs, dev):
        one.add_field(fc.prob, f)
    serve(warm, paced=False, srv=one)
    _, one_burst = serve(burst_reqs[:2000], paced=False, srv=one)
    one_rates = []
    for lam in (1000, 2000):
        reqs = request_stream(fcs, int(min(max_requests, lam * seconds_per_rate)), lam, seed=int(lam))
        _, st1 = serve(reqs, srv=one)
        st1["rate"] = lam
        one_rates.append(st1)
    one.close()
    plain_rate = len(sample) / plain_s
    return {
        "workload": "16 resident fields (15 of grid 32-160, nt 20-100, nrzns 200-2000, 4-8 modes; one "
                    "300x300x150, nrzns 2000, 8 modes), 8/16 headings per request, random start/target, "
                    "2% of requests on the large field; Poisson arrivals",
        "warmup_builds_s": round(warm_s, 3), "models_resident": st["models_resident"],
        "rates": per_rate, "burst": burst,
        "plain": {"sample": len(sample), "solves_per_s": round(plain_rate, 2),
                  "p50_ms": round(float(np.percentile(plain_lat, 50)), 3),
                  "p99_ms": round(float(np.percentile(plain_lat, 99)), 3)},
        "unbatched_server": {"max_batch": 1, "burst": one_burst, "rates": one_rates,
                             "note": "same server, cached base models, one request per launch"},
        "speedup_vs_plain_burst": round(burst["solves_per_s"] / plain_rate, 1),
        "batching_speedup_burst": round(burst["solves_per_s"] / one_burst["solves_per_s"], 2),
        "speedup_vs_plain_at_2000": round(per_rate[-1]["solves_per_s"] / plain_rate, 1),
        "max_rel_value_err_vs_plain": err,
        "server": {"batches": st["batches"], "models_built": st["models_built"],
                   "bytes_in_use": st["bytes_in_use"], "device_solve_ms": round(st["solve_ms"], 2)},
    }


def run_envgen() -> dict:
    """The environment generator at the reference script's parameters (25 x 25
    coarse grid interpolated 8x to 200 x 200, nt=10, 1000 realisations, 3
    modes): GPU time of e2e_env_generate, and the CPU restatement of the
    reference generator (pure-Python realisations, numpy SVD, scipy griddata)
    timed on two of the ten time steps and scaled to ten."""
    import torch

    from e2e_gpu_dp_b200 import envgen
    from oracle import envgen as OE

    cfg = envgen.reference_defaults()
    cfg["dyn_obstacle_data"] = ("None",)
    envgen.build_environment_DG_with_westward_clouds(**cfg)  # warm-up (library, solver handles)
    runs = []
    for _ in range(3):
        t0 = time.perf_counter()
        out = envgen.build_environment_DG_with_westward_clouds(device=True, **cfg)
        torch.cuda.synchronize()
        runs.append((time.perf_counter() - t0, out["stats"]["seconds"]))
    wall = statistics.median(r[0] for r in runs)
    dev = statistics.median(r[1] for r in runs)
    res = {"config": "init_gsize 25, interpolate_degree 8 (200x200), nt 10, n_wsamples 1000, n_modes 3",
           "device_s": round(dev, 4), "wall_s": round(wall, 4),
           "svals_vel_t1": [round(float(x), 6) for x in out["svals_vel"][1]]}
    sample = dict(cfg)
    sample.pop("op_nrzns")
    sample["nt"] = 2
    sample["n_modes"] = 2  # the reference asserts n_modes <= nt
    t0 = time.perf_counter()
    OE.generate(**sample)
    cpu_s = (time.perf_counter() - t0) * cfg["nt"] / sample["nt"]
    res.update({"cpu_restatement_s_extrapolated": round(cpu_s, 2), "cpu_sample": "2 of 10 time steps",
                "speedup_vs_cpu": round(cpu_s / wall, 1)})
    return res


def small_case_cpu(threads: int, trig=None):
    """The CPU-runnable workload in full on the host: the 50x50 grid, nt=30,
    8 headings, 500 realisations, 4 modes, 5 % obstacles, target (45, 25),
    built by the oracle port (the C restatement of the reference's builder)
    and solved by its FP64 backward induction, both timed on ``threads``
    threads.  Returns the timing, the problem, its fields, the oracle's model
    and its FP64 values."""
    from e2e_gpu_dp_b200.problem import config, make_fields
    from oracle import pyoracle as O

    prob, spec = config("c1", seed=1234)
    fields = make_fields(prob, spec)
    t0 = time.perf_counter()
    m = O.build_model(prob, fields, trig=trig, nthreads=threads)
    t1 = time.perf_counter()
    V64, _, _ = O.vi_f64_layers(prob.ncells, prob.nt, prob.num_actions, m["row_ptr"], m["col"], m["cnt"],
                                prob.nrzns, m["R_full"], nthreads=threads)
    t2 = time.perf_counter()
    return {"build_s": t1 - t0, "solve_s": t2 - t1, "threads": threads}, prob, fields, m, V64


def run_small_case(reps: int = 5) -> dict:
    """The CPU-runnable workload (50x50, nt=30, 8 headings, 500
    realisations): the oracle port on all host threads, in full, against the
    device's build + layered solve of the same seeded inputs (CUDA events,
    fields resident, after one warm-up), with the device's rows compared to
    the oracle's bit for bit and its values to the FP64 induction."""
    import torch

    from e2e_gpu_dp_b200 import api

    from e2e_gpu_dp_b200.problem import config

    threads = os.cpu_count() or 1
    # the oracle takes the device's cos/sin of the headings, so that the rows
    # can be compared bit for bit
    tab = api.action_table(config("c1", seed=1234)[0])
    cpu, prob, fields, om, V64 = small_case_cpu(threads, trig=(tab["cos"], tab["sin"]))
    stream = torch.cuda.current_stream()
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in fields.items()}
    V = torch.empty(prob.ns, dtype=torch.float32, device="cuda")
    pi = torch.empty(prob.ns, dtype=torch.int32, device="cuda")
    m = api.build_model(prob, dev, stream=stream)
    m.solve(method="layered", value=V, policy=pi, stream=stream)
    m.free()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        m = api.build_model(prob, dev, stream=stream)
        m.solve(method="layered", value=V, policy=pi, stream=stream)
        if _ < reps - 1:
            m.free()
    b.record(stream)
    torch.cuda.synchronize()
    gpu_s = a.elapsed_time(b) / 1e3 / reps
    h = m.to_host()
    m.free()
    same = (np.array_equal(h["row_ptr"], om["row_ptr"]) and np.array_equal(h["col"], om["col"])
            and np.array_equal(h["cnt"], om["cnt"]))
    Vh = V.cpu().numpy().astype(np.float64)
    scale = float(np.max(np.abs(V64)))
    cpu_s = cpu["build_s"] + cpu["solve_s"]
    return {"workload": "50x50 grid, nt=30, 8 headings, nrzns 500, 4 modes, 5% obstacles, target (45, 25)",
            "gpu_build_solve_s": round(gpu_s, 6), "gpu_reps": reps,
            "cpu_port_s": round(cpu_s, 3), "cpu_port_build_s": round(cpu["build_s"], 3),
            "cpu_port_solve_s": round(cpu["solve_s"], 3), "cpu_threads": threads,
            "cpu_kind": "oracle port (C restatement of the reference's builder, FP64 induction), in full",
            "speedup_vs_cpu": round(cpu_s / gpu_s, 1) if gpu_s > 0 else None,
            "rows_identical_to_oracle": bool(same),
            "max_rel_value_err_vs_fp64": float(np.max(np.abs(Vh - V64)) / scale) if scale > 0 else None}


def run_precision(sample_rows: int = 80000) -> dict:
    """Precision form: 300x300 grid, nt=150 (13.5 M states), 16 headings,
    nrzns 2000, 8 modes; uint16 counts with int32 next states, FP32 values, the
    FP64 Bellman residual of the verification sweep, and an FP64 backward solve
    on the GPU as the library's own check (max |V32 - V64| / max |V64|).  Then
    two checks that do not use the library: ``sample_rows`` rows built by the
    oracle against the device's, and an FP64 backward induction on the host
    (the oracle) over the device's model: value error and policy mismatches
    outside the FP64 tie band."""
    import torch

    from e2e_gpu_dp_b200 import api
    from e2e_gpu_dp_b200.problem import config
    from e2e_gpu_dp_b200.workloads import device_fields

    prob, spec = config("c3", seed=1234)
    dev = device_fields(prob, spec)
    stream = torch.cuda.current_stream()
    V = torch.empty(prob.ns, dtype=torch.float32, device="cuda")
    pi = torch.empty(prob.ns, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    m = api.build_model(prob, dev, count_type="u16", stream=stream)
    _, _, st = m.solve(method="layered", value=V, policy=pi, stream=stream)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    _, _, chk = m.solve(method="layered", fp64_check=True, value=V, policy=pi, stream=stream)
    inf = m.info()
    # independent checks on the host: the oracle's rows of 8 blocks spread over
    # the layers against the device's, bit for bit; an FP64 backward induction
    # (the oracle, on the host) over the device's model copied down: value error
    # and the policy's FP64 margin (actions more than the tie band below the
    # best are mismatches)
    from e2e_gpu_dp_b200.problem import make_fields
    from oracle import pyoracle as O

    threads = os.cpu_count() or 1
    h = m.to_host()
    m.free()
    fields = make_fields(prob, spec)
    tab = api.action_table(prob)
    n_rows = (prob.nt - 1) * prob.ncells * prob.num_actions
    per = sample_rows // 8
    blocks = []
    ts = time.perf_counter()
    for c in range(8):
        r0 = int((c + 0.5) * n_rows / 8) - per // 2
        blocks.append((r0, O.build_rows(prob, fields, trig=(tab["cos"], tab["sin"]), r0=r0, r1=r0 + per,
                                        nthreads=threads)))
    sample_s = time.perf_counter() - ts
    par = parity_sample(h, blocks)
    del blocks, fields
    tf = time.perf_counter()
    V64, _, gap = O.vi_f64_layers(prob.ncells, prob.nt, prob.num_actions, h["row_ptr"], h["col"],
                                  h["cnt"], prob.nrzns, h["R"], policy=pi.cpu().numpy(),
                                  nthreads=threads)
    f64_s = time.perf_counter() - tf
    scale = float(np.max(np.abs(V64)))
    band = 2e-5 * max(1.0, scale)
    Vh = V.cpu().numpy().astype(np.float64)
    host_check = {"kind": "oracle/e2e_oracle.c FP64 backward induction on the host over the device's model",
                  "threads": threads, "seconds": round(f64_s, 2),
                  "max_abs_err": float(np.max(np.abs(Vh - V64))),
                  "max_rel_err": float(np.max(np.abs(Vh - V64)) / scale),
                  "policy_mismatches_outside_ties": int(np.sum(gap > band)),
                  "policy_differs_within_ties": int(np.sum((gap > 0) & (gap <= band))),
                  "tie_band": band}
    del h, V64, gap
    return {"workload": "300x300 grid, nt=150, 16 headings, nrzns 2000, 8 modes, uint16 counts",
            "states": prob.ns, "rows": inf["n_rows"], "nnz": inf["nnz"],
            "count_type": "u16" if inf["count_type"] == 0 else inf["count_type"],
            "index_bits": inf["index_bits"], "build_kernel_ms": round(inf["build_kernel_ms"], 2),
            "pack_ms": round(st["pack_ms"], 2), "solve_ms": round(st["seconds"] * 1e3, 3),
            "layered_pass_ms": round(st["sweep_seconds"] * 1e3, 3), "build_solve_wall_s": round(wall, 3),
            "fp64_residual": chk["residual"], "fp64_max_abs_err": chk["fp64_max_abs_err"],
            "fp64_max_rel_err": chk["fp64_max_rel_err"],
            "fp64_oracle": host_check,
            "parity_sample": {**par, "oracle_s": round(sample_s, 2), "threads": threads}}


def run_reference(args, ws, rank, local):
    if rank != 0:
        return None
    from oracle import run_ref
    from e2e_gpu_dp_b200.problem import config, make_fields

    if not (run_ref.have_reference(WORKLOAD) and run_ref.have_reference("t_time")):
        return {"impl": "reference", "unavailable": "reference binaries not built into oracle/_ref "
                "(python oracle/build_ref.py needs the reference sources)"}
    prob, spec = config(WORKLOAD, seed=1234)
    fields = make_fields(prob, spec)
    work = tempfile.mkdtemp(prefix="e2e_ref_")
    try:
        for _ in range(args.warmup):  # process start, driver and binary warm-up on a small problem
            run_ref.run("t_time", os.path.join(work, "warm"), keep_model=False)
        runs = []
        with Clocks(local) as clk:
            clk.begin()
            for _ in range(args.steps):
                runs.append(run_ref.run(WORKLOAD, os.path.join(work, "c2"), prob=prob, fields=fields,
                                        keep_model=False))
                clk.tick()
        clocks = clk.summary()
    finally:
        subprocess.run(["rm", "-rf", work])
    wall = [r["wall_build_s"] + r["wall_convert_s"] + r["wall_solve_s"] for r in runs]
    value = statistics.mean(wall)
    return {
        "impl": "reference",
        "metric": "build+VI sec",
        "value": round(value, 4),
        "unit": "s",
        "n_gpus": 1,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(value * 1e3, 1),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "fp32",
        "data": "synthetic (same seeded inputs as the ours arm)",
        "config": workload_config(prob, 1),
        "pipeline": "build_model -> convert -> spvi_2",
        "phases_s": {"build_loop": statistics.mean(r["build_loop_s"] for r in runs),
                     "build_process": statistics.mean(r["wall_build_s"] for r in runs),
                     "convert": statistics.mean(r["wall_convert_s"] for r in runs),
                     "solve_process": statistics.mean(r["wall_solve_s"] for r in runs),
                     "solve_total_reported": statistics.mean(r["solve_total_s"] or 0 for r in runs),
                     "iterations": runs[-1]["iterations"]},
        "cpu_baseline": {"value": round(value, 4), "unit": "s", "cores": 1, "kind": "reference",
                         "sample": "the reference's own CUDA programs (compiled unmodified for sm_100a) "
                                   "on the full workload, one host thread driving the GPU, wall clock "
                                   "of build_model + int32 convert + spvi_2"},
        "e2e": {"value": round(value, 4), "unit": "s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "clocks": clocks,
    }


def profile_case():
    """Small case of the same kernels for ncu: the workload's grid, headings,
    realisations and modes with nt=30 (fields 0.1 GB, model 0.4 GB > L2); one
    build and one Jacobi solve (30 sweeps of the fused VI kernel)."""
    import dataclasses

    import torch

    from e2e_gpu_dp_b200 import api
    from e2e_gpu_dp_b200.problem import config, make_fields

    prob, spec = config(WORKLOAD, seed=1234)
    prob = dataclasses.replace(prob, nt=30)
    fields = make_fields(prob, spec)
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in fields.items()}
    m = api.build_model(prob, dev)
    _, _, st = m.solve(method="jacobi", threshold=0.1)
    inf = m.info()
    print(json.dumps({"profile_case": "c2 geometry, nt=30", "nnz": inf["nnz"], "rows": inf["n_rows"],
                      "build_kernel_ms": inf["build_kernel_ms"], "jacobi_sweeps": st["iterations"],
                      "bytes_per_sweep": st["bytes_per_sweep"],
                      "stream_bytes_per_sweep": st["stream_bytes_per_sweep"], "pack_ms": st["pack_ms"],
                      "jacobi_s": st["seconds"]}))
    m.free()
    return 0


def profile_batch():
    """Small case of the batched sweep for ncu: 32 of the batched form's
    problems with grid <= 96 (a few GB on the device), built, then solved in
    one direct launch with a fixed schedule (one warp per chunk, lean kernel,
    no prefetch)."""
    import torch

    from e2e_gpu_dp_b200 import api
    from e2e_gpu_dp_b200.workloads import batch_instances, device_fields

    insts = [x for x in batch_instances(256) if x.prob.gsize <= 96][:32]
    fields = [device_fields(x.prob, x.spec) for x in insts]
    models = api.build_models([x.prob for x in insts], fields)
    outs = [(torch.empty(x.prob.ns, dtype=torch.float32, device="cuda"),
             torch.empty(x.prob.ns, dtype=torch.int32, device="cuda")) for x in insts]
    sch = 1 | (4 << 4) | 0x100 | 0x200
    st = api.solve_batch(models, [o[0] for o in outs], [o[1] for o in outs], schedule=sch)
    st = api.solve_batch(models, [o[0] for o in outs], [o[1] for o in outs], schedule=sch)
    print(json.dumps({"profile_batch": len(insts), "rows": int(sum((x.prob.nt - 1) * x.prob.ncells *
                                                                    x.prob.num_actions for x in insts)),
                      "stream_bytes": st["stream_bytes"], "seconds": st["seconds"]}))
    for m in models:
        m.free()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 10; the reference arm, 42 s a step, 3)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-case", action="store_true", help="small case for ncu captures")
    ap.add_argument("--profile-batch", action="store_true", help="small batched case for ncu captures")
    ap.add_argument("--batched-only", action="store_true", help="only the batched form (256 uneven MDPs)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched form")
    ap.add_argument("--served-only", action="store_true", help="only the served form (request server)")
    ap.add_argument("--precision-only", action="store_true", help="only the precision form (300x300x150)")
    ap.add_argument("--no-precision", action="store_true", help="skip the precision form")
    ap.add_argument("--no-served", action="store_true", help="skip the served form")
    ap.add_argument("--envgen-only", action="store_true", help="only the environment generator")
    ap.add_argument("--no-envgen", action="store_true", help="skip the environment generator")
    ap.add_argument("--no-small-case", action="store_true",
                    help="skip the 50x50 CPU-runnable workload (oracle port in full vs the device)")
    args = ap.parse_args()
    if args.profile_case:
        return profile_case()
    if args.profile_batch:
        return profile_batch()
    if args.batched_only:
        print(json.dumps({"batched": run_batched()}), flush=True)
        return 0
    if args.served_only:
        print(json.dumps({"served": run_served()}), flush=True)
        return 0
    if args.precision_only:
        print(json.dumps({"precision": run_precision()}), flush=True)
        return 0
    if args.envgen_only:
        print(json.dumps({"envgen": run_envgen()}), flush=True)
        return 0
    ws, rank, local = _dist()
    if args.steps is None:
        args.steps = 3 if args.impl == "reference" else 10
    if args.impl == "reference":
        out = run_reference(args, ws, rank, local)
        if out is not None:
            print(json.dumps(out), flush=True)
        return 0
    if ws > 1:
        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    try:
        line = run_ours(args, ws, rank, local)
        if rank == 0 and ws == 1 and not args.no_batched:
            line["batched"] = run_batched()
        if rank == 0 and ws == 1 and not args.no_served:
            line["served"] = run_served()
        if rank == 0 and ws == 1 and not args.no_precision:
            line["precision"] = run_precision()
        if rank == 0 and ws == 1 and not args.no_envgen:
            line["envgen"] = run_envgen()
        if rank == 0 and ws == 1 and not args.no_cpu_baseline and not args.no_small_case:
            try:
                line["small_case"] = run_small_case()
            except Exception as e:  # an auxiliary figure never costs the bench line
                line["small_case"] = {"error": repr(e)[:300]}
        if rank == 0:
            print(json.dumps(line), flush=True)
    finally:
        if ws > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
