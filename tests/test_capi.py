"""The C-ABI library loads on a CPU-only host and exports every declared entry point;
pure-host sizing calls work and reject bad arguments (no kernel launches here)."""

import ctypes as C
import os
import re

import pytest

from genesis_b200 import _native as nat
from genesis_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"^\s*int\s+(mpm_\w+)\s*\(", txt, flags=re.M))
    return names


@pytest.fixture(scope="module")
def lib():
    B.build()
    return nat.load()


def test_every_declared_symbol_is_exported_and_bound(lib):
    declared = _declared()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
        assert name in nat.SIGNATURES, f"{name} has no ctypes binding"


def test_abi_and_struct_layout(lib):
    assert lib.mpm_abi_version() == nat.ABI_VERSION
    sizes = (C.c_int32 * 7)()
    assert lib.mpm_struct_sizes(sizes) == 0
    assert tuple(sizes) == (C.sizeof(nat.Instance), C.sizeof(nat.Material), C.sizeof(nat.Problem),
                            C.sizeof(nat.Particles), C.sizeof(nat.Tables), C.sizeof(nat.Collider),
                            C.sizeof(nat.ForceField))


def _prob(n=1000, nb=512, P=256):
    mc = C.c_int32()
    assert nat.load().mpm_max_chunks(n, nb, P, C.byref(mc)) == 0
    return nat.Problem(n_instances=1, n_particles=n, n_blocks=nb, n_materials=1, chunk_particles=P,
                       max_chunks=mc.value, grid_ctas=0, flags=0)


def test_workspace_sizing(lib):
    p = _prob()
    out = C.c_uint64()
    assert lib.mpm_workspace_bytes(C.byref(p), C.byref(out)) == 0
    # at least the two block-major float4 grids
    assert out.value >= 2 * 512 * 64 * 16
    mm, gv = C.c_uint64(), C.c_uint64()
    assert lib.mpm_grid_offsets(C.byref(p), C.byref(mm), C.byref(gv)) == 0
    assert mm.value % 256 == 0 and gv.value % 256 == 0 and gv.value >= mm.value + 512 * 64 * 16


def test_max_chunks_bound(lib):
    mc = C.c_int32()
    assert lib.mpm_max_chunks(500_000, 35937, 256, C.byref(mc)) == 0
    assert mc.value == 500_000 // 256 + 35937 + 1


def test_invalid_arguments_rejected(lib):
    out = C.c_uint64()
    p = _prob()
    p.chunk_particles = 100  # not one of 128/256/512
    assert lib.mpm_workspace_bytes(C.byref(p), C.byref(out)) == nat.MPM_E_INVALID
    p = _prob()
    p.max_chunks = 1
    assert lib.mpm_workspace_bytes(C.byref(p), C.byref(out)) == nat.MPM_E_INVALID
    p = _prob()
    p.n_blocks = 1 << 40
    assert lib.mpm_workspace_bytes(C.byref(p), C.byref(out)) in (nat.MPM_E_CAPACITY, nat.MPM_E_INVALID)
    assert lib.mpm_workspace_bytes(None, C.byref(out)) == nat.MPM_E_INVALID
    assert lib.mpm_graph_launch(None, None) == nat.MPM_E_INVALID
    assert lib.mpm_graph_destroy(None) == nat.MPM_E_INVALID


def test_missing_library_fails_loudly(tmp_path):
    with pytest.raises(nat.NativeLibraryError):
        # a fresh loader on a path that does not exist must raise, never fall back
        saved = nat._lib
        try:
            nat._lib = None
            nat.load(str(tmp_path / "nope.so"))
        finally:
            nat._lib = saved


def test_block_count_above_the_scan_limit_is_refused(lib):
    """More grid blocks than the single-pass scan covers (4096 x 4096) -> MPM_E_CAPACITY."""
    mc = C.c_int32()
    assert lib.mpm_max_chunks(1000, 4096 * 4096, 128, C.byref(mc)) == 0
    ok = nat.Problem(n_instances=1, n_particles=1000, n_blocks=4096 * 4096, n_materials=1, chunk_particles=128,
                     max_chunks=mc.value, grid_ctas=0, flags=0)
    b = C.c_uint64()
    assert lib.mpm_workspace_bytes(C.byref(ok), C.byref(b)) == 0
    assert lib.mpm_max_chunks(1000, 4096 * 4096 + 1, 128, C.byref(mc)) == 0
    big = nat.Problem(n_instances=1, n_particles=1000, n_blocks=4096 * 4096 + 1, n_materials=1, chunk_particles=128,
                      max_chunks=mc.value, grid_ctas=0, flags=0)
    assert lib.mpm_workspace_bytes(C.byref(big), C.byref(b)) == nat.MPM_E_CAPACITY
