"""The recorded reverse pass (mpm_substeps_record + mpm_substeps_adjoint_recorded) against the
per-substep adjoint that recomputes each substep's grid itself (mpm_substep_adjoint), through
the C ABI, on the benchmark's four-material mix with per-particle E.

Given the same input states, the two differ only in where the forward grid comes from:
recorded by the forward that produced the states, or recomputed from the state by the adjoint
call, which can round the grid's float reductions in another order.  Tolerance: 1e-4 of the largest entry of each
adjoint channel group after 10 substeps (the rollout gradients themselves are checked against
float64 references in test_gpu_grad*.py)."""

import ctypes as C

import numpy as np
import pytest
import torch

from genesis_b200 import _native as nat

pytestmark = pytest.mark.gpu


def _mixed_desc(T=10):
    """Four 6^3 blocks (Liquid, Sand, Snow, ElastoPlastic) with per-particle E (log-normal,
    sigma 0.5) thrown at the floor of a 32^3 grid."""
    from genesis_b200 import workloads as W

    blocks = [("liquid", dict(E=1e5, nu=0.2), (0.1, 0.1)), ("sand", dict(E=1e5, friction_angle=45), (0.3, 0.1)),
              ("snow", dict(E=1e5, yield_lower=2.5e-2, yield_higher=7.5e-3), (0.1, 0.3)),
              ("elastoplastic", dict(E=1e5, von_mises_yield_stress=1e4), (0.3, 0.3))]
    rng = np.random.default_rng(7)
    dx = 1.0 / 32
    pos, mat, E = [], [], []
    for mi, (kind, kw, xy) in enumerate(blocks):
        lat = W.jittered_lattice(rng, 6, (xy[0], xy[1], 3 * dx + 0.0012), 0.5 * dx)
        pos.append(lat)
        mat.append(np.full(len(lat), mi))
        E.append(kw["E"] * np.exp(0.5 * rng.normal(size=len(lat))))
    pos = np.concatenate(pos)
    n = len(pos)
    return W.SceneDesc(name="recorded_adjoint", grid_density=32, particle_size=0.5 * dx, dt=2e-4, n_substeps=T,
                       pos=pos, vel=np.tile([0.4, -0.2, -1.0], (n, 1)), mat_idx=np.concatenate(mat),
                       materials=[(k, dict(kw)) for k, kw, _ in blocks], upper_bound=(0.5, 0.5, 0.5),
                       E_particle=np.concatenate(E))


def _runtime(d):
    from genesis_b200.engine.runtime import runtime_from_descs

    rt = runtime_from_descs([d], sort_interval=0, use_graphs=False)
    E = torch.as_tensor(d.E_particle, dtype=torch.float32, device=rt.device)
    nu = torch.tensor([0.2, 0.3, 0.3, 0.3], device=rt.device)[torch.as_tensor(d.mat_idx, device=rt.device)]
    mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
    rt.set_lame(mu, lam)
    rt.ensure_sorted()
    return rt


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream or None)


def test_record_and_recorded_adjoint_match_the_per_substep_adjoint():
    d = _mixed_desc()
    m = d.n_substeps
    rt = _runtime(d)
    lib = rt.lib
    start = rt.state.clone()
    nb = C.c_uint64()
    nat.check("mpm_adjoint_workspace_bytes", lib.mpm_adjoint_workspace_bytes(C.byref(rt.prob), C.byref(nb)))
    aws = torch.empty(int(nb.value), dtype=torch.uint8, device=rt.device)
    gb = C.c_uint64()
    nat.check("mpm_record_grid_bytes", lib.mpm_record_grid_bytes(C.byref(rt.prob), C.byref(gb)))

    # recorded forward: the states it stores are the per-substep states of an ordinary run
    rec_state = torch.empty((m,) + tuple(rt.state.shape), dtype=torch.float32, device=rt.device)
    rec_grid = torch.empty(m * int(gb.value), dtype=torch.uint8, device=rt.device)
    nat.check("mpm_substeps_record", lib.mpm_substeps_record(
        C.byref(rt.prob), C.byref(rt.tables), C.byref(rt.par), rt._ws, m, C.c_void_p(rec_state.data_ptr()),
        C.c_void_p(rec_grid.data_ptr()), _stream()))
    recorded_end = rt.state.clone()
    rt.state.copy_(start)
    states = []
    for _ in range(m):
        states.append(rt.state.clone())
        rt.substeps(1)
    n = rt.n
    groups = {"x": slice(0, 3), "v": slice(3, 6), "C": slice(6, 15), "F": slice(15, 24), "Jp": slice(24, 25)}

    def close(a, b, j):
        # the grid's float reductions may round in another order from run to run: each channel
        # group within 1e-4 of its largest entry, positions within 1e-5 m
        for name, sl in groups.items():
            d = (a[sl, :n] - b[sl, :n]).abs().max().item()
            bound = 1e-5 if name == "x" else 1e-4 * max(b[sl, :n].abs().max().item(), 1e-30)
            assert d <= bound, (j, name, d, bound)

    for j in range(m):
        close(rec_state[j], states[j], j)
    close(recorded_end, rt.state, m)
    assert rt.status() == 0

    # the same output adjoint through both reverse passes
    g = torch.Generator(device="cpu").manual_seed(3)
    seed = torch.randn(rt.state.shape, generator=g).to(rt.device)
    seed[:, n:] = 0
    adj_a, adj_b = seed.clone(), seed.clone()
    lb_a = torch.zeros((3, rt.stride), dtype=torch.float32, device=rt.device)
    lb_b = torch.zeros_like(lb_a)
    for j in range(m - 1, -1, -1):
        # the same input states as the recorded pass (a second forward run rounds its grid
        # reductions in another order, which the plastic return mappings' branches amplify)
        par = nat.Particles.from_buffer_copy(rt.par)
        par.state = rec_state[j].data_ptr()
        nat.check("mpm_substep_adjoint", lib.mpm_substep_adjoint(
            C.byref(rt.prob), C.byref(rt.tables), C.byref(par), C.c_void_p(adj_a.data_ptr()),
            C.c_void_p(lb_a.data_ptr()), rt._ws, C.c_void_p(aws.data_ptr()), _stream()))
    # in two calls, as a trajectory loss splits it
    for first, count in ((4, m - 4), (0, 4)):
        nat.check("mpm_substeps_adjoint_recorded", lib.mpm_substeps_adjoint_recorded(
            C.byref(rt.prob), C.byref(rt.tables), C.byref(rt.par), first, count, C.c_void_p(rec_state.data_ptr()),
            C.c_void_p(rec_grid.data_ptr()), C.c_void_p(adj_b.data_ptr()), C.c_void_p(lb_b.data_ptr()),
            C.c_void_p(aws.data_ptr()), _stream()))
    torch.cuda.synchronize()
    for name, sl in groups.items():
        a, b = adj_a[sl, :n], adj_b[sl, :n]
        scale = max(a.abs().max().item(), 1e-30)
        err = (a - b).abs().max().item() / scale
        print(f"\n[recorded adjoint] {name}: max rel. difference {err:.1e}")
        assert err <= 1e-4, (name, err)
    for r in range(2):
        a, b = lb_a[r, :n], lb_b[r, :n]
        assert (a - b).abs().max().item() <= 1e-4 * max(a.abs().max().item(), 1e-30), r


def test_recorded_calls_refuse_colliders_and_bad_ranges():
    d = _mixed_desc()
    rt = _runtime(d)
    lib = rt.lib
    rec = torch.empty(16, dtype=torch.float32, device=rt.device)
    adj = torch.zeros_like(rt.state)
    lb = torch.zeros((3, rt.stride), dtype=torch.float32, device=rt.device)
    rc = lib.mpm_substeps_adjoint_recorded(C.byref(rt.prob), C.byref(rt.tables), C.byref(rt.par), -1, 1,
                                           C.c_void_p(rec.data_ptr()), C.c_void_p(rec.data_ptr()),
                                           C.c_void_p(adj.data_ptr()), C.c_void_p(lb.data_ptr()),
                                           C.c_void_p(rec.data_ptr()), _stream())
    assert rc == nat.MPM_E_INVALID
    tab = nat.Tables.from_buffer_copy(rt.tables)
    cols = (nat.Collider * 1)()
    tab.colliders = C.cast(cols, C.c_void_p)
    tab.n_colliders = 1
    rc = lib.mpm_substeps_record(C.byref(rt.prob), C.byref(tab), C.byref(rt.par), rt._ws, 1,
                                 C.c_void_p(rec.data_ptr()), C.c_void_p(rec.data_ptr()), _stream())
    assert rc == nat.MPM_E_INVALID
