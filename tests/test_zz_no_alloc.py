"""The allocation-free entry point, mpm_substeps_noalloc, called through the C ABI.

Some callers can't allocate device memory: host applications whose allocator reserves
the GPU up front, and plugin hosts that forbid cudaMalloc.  For them the library keeps
its workspace in a static device array.  This file checks that two calls in a row give
the same state as the ordinary entry point with a caller-allocated workspace and as the
float64 oracle, that the NaN check reaches such a caller through mpm_noalloc_status, and
that oversized problems are refused before any work is queued.  It is named so that pytest
collects it last.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from genesis_b200 import _native as nat
from genesis_b200 import workloads as W


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream or None)


def _state(rt):
    st = rt.get_state(("pos", "vel", "C", "F", "Jp"))
    torch.cuda.synchronize()
    return {k: v.cpu().numpy() for k, v in st.items()}


@pytest.mark.gpu
def test_noalloc_matches_workspace_entry_point_on_two_calls():
    from genesis_b200.engine.runtime import runtime_from_descs

    d = W.elastic_cube(n_side=16)
    d.vel = np.random.default_rng(11).normal(0.0, 0.5, size=d.vel.shape)
    ref = runtime_from_descs([d], use_graphs=False)  # owns a caller-allocated workspace
    noa = runtime_from_descs([d], use_graphs=False)  # only its particle buffers and tables are used
    lib = nat.load()
    need = C.c_uint64()
    assert lib.mpm_workspace_bytes(C.byref(noa.prob), C.byref(need)) == 0
    assert need.value <= nat.NOALLOC_SCRATCH_BYTES
    n, K = 20, 8
    for call in range(2):
        first = call * n
        rc = lib.mpm_substeps(C.byref(ref.prob), C.byref(ref.tables), C.byref(ref.par), ref._ws, n, K, first, _stream())
        assert rc == 0
        rc = lib.mpm_substeps_noalloc(C.byref(noa.prob), C.byref(noa.tables), C.byref(noa.par), n, K, first, _stream())
        assert rc == 0
        a, b = _state(ref), _state(noa)
        # same tolerance as the other GPU parity tests: float32 atomics sum in any order
        assert np.abs(a["pos"] - b["pos"]).max() <= 1e-6, call
        assert np.abs(a["vel"] - b["vel"]).max() <= 1e-4 * max(1.0, np.abs(a["vel"]).max()), call
        assert np.abs(a["F"] - b["F"]).max() <= 1e-5, call
        assert np.abs(a["Jp"] - b["Jp"]).max() <= 1e-6, call
    assert ref.status() == 0
    word, inst = C.c_uint32(7), (C.c_uint32 * 1)(7)
    assert lib.mpm_noalloc_status(C.byref(noa.prob), 0, C.byref(word), inst, _stream()) == 0
    assert word.value == 0 and inst[0] == 0
    # the allocation-free run against the float64 oracle, 2 x 20 substeps from the same start
    from oracle import bridge, cref

    want, rc = cref.substeps(*bridge.from_desc(d, np.float64), 2 * n)
    assert rc == 0
    assert np.abs(b["pos"] - want["x"]).max() <= 1e-5


@pytest.mark.gpu
def test_noalloc_status_reports_a_nan_position():
    """A NaN position planted on the host sets MPM_STATUS_NAN in the word the caller reads back
    through mpm_noalloc_status; clearing resets it, and the next call starts from zero."""
    from genesis_b200.engine.runtime import runtime_from_descs

    d = W.elastic_cube(n_side=8)
    noa = runtime_from_descs([d], use_graphs=False)
    pos = d.pos.copy()
    pos[3] = np.nan
    noa.set_state(pos=pos)
    lib = nat.load()
    assert lib.mpm_substeps_noalloc(C.byref(noa.prob), C.byref(noa.tables), C.byref(noa.par), 2, 8, 0,
                                    _stream()) == 0
    word, inst = C.c_uint32(0), (C.c_uint32 * 1)(0)
    assert lib.mpm_noalloc_status(C.byref(noa.prob), 1, C.byref(word), inst, _stream()) == 0
    assert word.value & nat.MPM_STATUS_NAN and inst[0] & nat.MPM_STATUS_NAN
    assert lib.mpm_noalloc_status(C.byref(noa.prob), 0, C.byref(word), inst, _stream()) == 0
    assert word.value == 0 and inst[0] == 0
    # a clean problem after it: the next call clears the array, so its word reads 0
    clean = runtime_from_descs([W.elastic_cube(n_side=8)], use_graphs=False)
    assert lib.mpm_substeps_noalloc(C.byref(clean.prob), C.byref(clean.tables), C.byref(clean.par), 2, 8, 0,
                                    _stream()) == 0
    assert lib.mpm_noalloc_status(C.byref(clean.prob), 0, C.byref(word), None, _stream()) == 0
    assert word.value == 0


def test_noalloc_refuses_problems_larger_than_its_scratch():
    lib = nat.load()
    n, nb, P = 4_000_000, 300_000, 128
    mc = C.c_int32()
    assert lib.mpm_max_chunks(n, nb, P, C.byref(mc)) == 0
    prob = nat.Problem(n_instances=1, n_particles=n, n_blocks=nb, n_materials=1, chunk_particles=P,
                       max_chunks=mc.value, grid_ctas=0, flags=0)
    need = C.c_uint64()
    assert lib.mpm_workspace_bytes(C.byref(prob), C.byref(need)) == 0
    assert need.value > nat.NOALLOC_SCRATCH_BYTES
    par = nat.Particles(state=1, state_stride=n, mat=1, pflags=1, gid=1, slot=1, mu_p=None, lam_p=None)
    tab = nat.Tables(1, 1)  # never dereferenced: the size check comes first
    rc = lib.mpm_substeps_noalloc(C.byref(prob), C.byref(tab), C.byref(par), 1, 8, 0, None)
    assert rc == nat.MPM_E_CAPACITY
    word = C.c_uint32()
    assert lib.mpm_noalloc_status(C.byref(prob), 0, C.byref(word), None, None) == nat.MPM_E_CAPACITY
