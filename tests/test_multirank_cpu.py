"""The N > 1 plumbing of bench.py on CPU: two gloo ranks (the GPU runs use one
process per GPU over NCCL with the same helpers).  The workload is replicas:
no data-path collective, only the barrier around the timed region and the
max over ranks of the step time."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        w, r, loc = bench._dist()
        bench._barrier(w)
        step_ms = 100.0 + 50.0 * r          # the slower rank sets the step time
        m = bench._max_over_ranks(step_ms, w)
        value = bench.whole_job_seconds_per_solve(m, w)
        ref = bench.run_reference(None, w, r, loc) if r != 0 else "rank0"
        out[r] = (w, r, loc, m, value, ref)
        bench._barrier(w)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_replicas():
    ws = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank_main, args=(ws, port, out), nprocs=ws, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r, (w, rr, loc, m, value, ref) in res.items():
        assert (w, rr, loc) == (2, r, r)
        assert m == 150.0                    # max over ranks, seen by every rank
        assert value == pytest.approx(0.075)  # 2 solves per 150 ms step
    assert res[1][5] is None                 # reference arm: ranks > 0 do no work


def test_single_rank_needs_no_process_group():
    assert bench._dist() == (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
                             int(os.environ.get("LOCAL_RANK", "0")))
    assert bench._max_over_ranks(3.5, 1) == 3.5
    assert bench.whole_job_seconds_per_solve(500.0, 1) == 0.5
