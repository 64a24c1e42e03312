"""The C ABI from a C host: tests/c/abi_check.c compiled with gcc against
include/genesis_b200_mpm.h and linked to the built library (no GPU calls)."""

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc not available")
def test_c_host_builds_and_passes(tmp_path):
    from genesis_b200 import build

    lib = build.build()
    exe = tmp_path / "abi_check"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c", "abi_check.c"), "-o", str(exe),
                    "-L", os.path.dirname(lib), "-lgenesis_b200_mpm", "-Wl,-rpath," + os.path.dirname(lib)],
                   check=True, capture_output=True, text=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.count("ok ") == 8
