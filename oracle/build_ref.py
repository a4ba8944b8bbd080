"""Recipe: compile the reference's own CUDA programs into ``oracle/_ref/``.

ORACLE -- test infrastructure only.

The reference's builder takes its whole problem definition from
``input_to_build_model.h``, which ``main`` includes with a quoted ``#include``
*inside its body* (``src/build_model.cu:932``).  A quoted include resolves in
the directory of the including file first, so for each problem this recipe
makes ``oracle/_ref/<name>/`` holding a *symlink* ``build_model.cu`` to the
reference source and a generated ``input_to_build_model.h``; the compiler then
reads the reference source where it lies and the header beside the symlink.
No reference source is copied.

``src/spvi_2.cu`` is compiled where it lies, with
``-DCUSPARSE_MV_ALG_DEFAULT=CUSPARSE_SPMV_ALG_DEFAULT`` (that enumerator was
removed in CUDA 12).  Both programs include ``"cnpy.h"``; the third-party cnpy
library is not installed, so ``oracle/ref_shim/cnpy.h`` (own .npy I/O with the
same API subset) is put on the include path instead of linking ``-lcnpy``.

Build flags follow ``src/Makefile:14,23`` with two changes: device code for
sm_100a (the reference Makefile names no architecture) and ``-O3`` for the
host code (the Makefile passes none), which only speeds the reference up.

The reference sources are found at ``$E2E_REFERENCE_SRC`` or, by default, in
``../reference/src`` relative to this repository's root.

Usage (in a container that has the reference sources):
    python oracle/build_ref.py            # default problem set
    python oracle/build_ref.py c1 t_time  # selected problems
The binaries travel with the repository snapshot; nothing here is needed at
run time on a machine without the reference.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# The reference's src/ directory: $E2E_REFERENCE_SRC, else a checkout named
# "reference" beside this repository's root.
REF_SRC = os.environ.get("E2E_REFERENCE_SRC",
                         os.path.join(os.path.dirname(ROOT), "reference", "src"))
OUT = os.path.join(HERE, "_ref")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
DEFAULT_PROBLEMS = ["t_time", "t_custom", "t_energy2", "t_wide", "c1", "c2", "t_m10", "t_m8", "t_m6", "t_half",
                    "t_energy1", "t_energy3"]

sys.path.insert(0, ROOT)


def available() -> bool:
    return os.path.isfile(os.path.join(REF_SRC, "build_model.cu")) and os.path.isfile(
        os.path.join(REF_SRC, "spvi_2.cu"))


def _run(cmd):
    print("+", " ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_builder(name: str, prob) -> str:
    d = os.path.join(OUT, name)
    os.makedirs(d, exist_ok=True)
    link = os.path.join(d, "build_model.cu")
    if os.path.islink(link) or os.path.exists(link):
        os.remove(link)
    os.symlink(os.path.join(REF_SRC, "build_model.cu"), link)
    with open(os.path.join(d, "input_to_build_model.h"), "w") as fh:
        fh.write(prob.reference_header())
    exe = os.path.join(d, "build_model")
    _run([NVCC, *ARCH, "-O3", "-std=c++17", "-I", os.path.join(HERE, "ref_shim"), "-o", exe,
          link, "-w"])
    os.remove(link)
    return exe


def build_solver() -> str:
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, "spvi_2")
    _run([NVCC, *ARCH, "-O3", "-std=c++17", "-I", os.path.join(HERE, "ref_shim"),
          "-DCUSPARSE_MV_ALG_DEFAULT=CUSPARSE_SPMV_ALG_DEFAULT", "-o", exe,
          os.path.join(REF_SRC, "spvi_2.cu"), "-lcusparse", "-w"])
    return exe


def main(names):
    from e2e_gpu_dp_b200.problem import config

    if not available():
        print(f"reference sources not found under {REF_SRC}; nothing built")
        return 0
    build_solver()
    for n in names:
        prob, _ = config(n)
        build_builder(n, prob)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:] or DEFAULT_PROBLEMS))
