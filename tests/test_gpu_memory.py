"""Device memory of the library: the large-block cache and the host phase trace.

Blocks of 8 MiB and more that the library frees are kept and handed to the
next request of about the same size after an event wait on the freeing stream;
e2e_memory_trim returns them.  Builds and solves of different problems in any
order, on different streams, and after a trim, must give the same model, values
and policy as the first build of each problem.  With E2E_TRACE=1 each build and
solve prints one line of host phase timings.
"""
import hashlib
import os
import subprocess
import sys

import numpy as np
import pytest

from e2e_gpu_dp_b200 import _lib, api
from tests.helpers import problem

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _digest(prob, fields, stream=None):
    m = api.build_model(prob, fields, stream=stream)
    h = m.to_host()
    V, pi, _ = m.solve(method="layered", stream=stream)
    m.free()
    parts = [np.ascontiguousarray(h[k]).tobytes() for k in ("row_ptr", "col", "cnt", "R")]
    parts += [V.tobytes(), pi.tobytes()]
    return hashlib.sha1(b"".join(parts)).hexdigest()


def test_interleaved_sizes_and_trim_reproduce_first_build():
    names = ["c1", "t_wide", "t_custom"]
    cases = {n: problem(n) for n in names}
    first = {n: _digest(*cases[n]) for n in names}
    # blocks of one problem's sizes now serve the others (within a quarter of the size)
    for n in ["t_wide", "c1", "c1", "t_custom", "c1"]:
        assert _digest(*cases[n]) == first[n], n
    _lib.check(_lib.lib().e2e_memory_trim())
    assert _digest(*cases["c1"]) == first["c1"]


def test_blocks_freed_on_one_stream_reused_on_another():
    torch = pytest.importorskip("torch")
    prob, fields = problem("c1")
    ref = _digest(prob, fields)
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in fields.items()}
    torch.cuda.synchronize()
    m = api.build_model(prob, dev, stream=s1)
    m.free()  # model blocks freed on the legacy stream, taken by the build on s2
    assert _digest(prob, dev, stream=s2) == ref
    assert _digest(prob, dev, stream=s1) == ref


def test_trace_prints_host_phases():
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "from e2e_gpu_dp_b200 import api\n"
        "from tests.helpers import problem\n"
        "prob, f = problem('t_custom')\n"
        "m = api.build_model(prob, f)\n"
        "m.solve(method='layered')\n"
        "m.free()\n" % ROOT)
    env = dict(os.environ, E2E_TRACE="1")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stderr.splitlines() if ln.startswith("e2e_trace ")]
    build = [ln for ln in lines if ln.startswith("e2e_trace build_model ")]
    solve = [ln for ln in lines if ln.startswith("e2e_trace spvi_solve ")]
    assert len(build) == 1 and len(solve) == 1, lines
    for key in ("wall=", "cpu=", "vcsw=", "pool_mb=", " build=", " model_alloc=", " assemble="):
        assert key in build[0], (key, build[0])
    for key in (" pack=", " solve=", " outputs="):
        assert key in solve[0], (key, solve[0])
