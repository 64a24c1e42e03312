"""In-tree build of the sm_100a shared library ``libgenesis_b200_mpm.so``.

    python -m genesis_b200.build            # build if sources are newer than the .so
    python -m genesis_b200.build --force    # always rebuild
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
SOURCES = [os.path.join(CSRC, "mpm_kernels.cu")]
DEPS = SOURCES + [
    os.path.join(CSRC, "svd3.cuh"),
    os.path.join(CSRC, "constitutive.cuh"),
    os.path.join(CSRC, "mpm_adjoint.cuh"),
    os.path.join(ROOT, "include", "genesis_b200_mpm.h"),
]
OUT = os.path.join(HERE, "libgenesis_b200_mpm.so")

NVCC_FLAGS = [
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-O3",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-shared",
    "-cudart",
    "static",
]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build genesis_b200")
    return cand


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in DEPS if os.path.exists(d))


def build(force: bool = False, verbose: bool = False, extra_flags: list[str] | None = None) -> str:
    if not force and up_to_date():
        return OUT
    cmd = [nvcc_path(), *NVCC_FLAGS, *(extra_flags or []), "-o", OUT + ".tmp", *SOURCES]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose=True))
