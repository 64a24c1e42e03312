"""CUDA adjoint (checkpointed, behind torch.autograd) against the oracle adjoint and float64
central finite differences of the C restatement."""

import numpy as np
import pytest
import torch

from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _grads(d, checkpoint_every):
    from genesis_b200.grad import DifferentiableRollout, rollout

    sim = DifferentiableRollout(d, checkpoint_every=checkpoint_every)
    v0 = torch.tensor(d.meta["v0"], dtype=torch.float32, device="cuda", requires_grad=True)
    E = torch.tensor(d.E_particle, dtype=torch.float32, device="cuda", requires_grad=True)
    x = rollout(v0, E, sim)
    tgt = torch.tensor(d.meta["target"], dtype=torch.float32, device="cuda")
    loss = ((x.mean(0) - tgt) ** 2).sum()
    loss.backward()
    return float(loss.detach()), v0.grad.cpu().numpy().astype(np.float64), E.grad.cpu().numpy().astype(np.float64)


def test_adjoint_matches_oracle_adjoint_small():
    from oracle import bridge
    from oracle import mpm_adjoint as AD
    from oracle import mpm_ref as R

    d = W.diff_elastic(n=343, n_substeps=60)
    loss, gv, gE = _grads(d, checkpoint_every=20)
    p, mats, st = bridge.from_desc(d, np.float64)
    n = d.n_particles
    st["v"] = np.tile(d.meta["v0"], (n, 1))
    mass = np.full(n, R.particle_mass(p, mats[0]))
    l64, gv64, gE64, _ = AD.rollout_loss_and_grad(p, st, d.E_particle, 0.3, mass, d.n_substeps, d.meta["target"])
    assert abs(loss - l64) <= 1e-4 * l64
    assert np.abs(gv - gv64).max() <= 1e-2 * np.abs(gv64).max(), (gv, gv64)
    assert np.linalg.norm(gE - gE64) <= 5e-2 * np.linalg.norm(gE64), np.linalg.norm(gE - gE64) / np.linalg.norm(gE64)


def test_adjoint_full_config_against_fp64_finite_differences():
    """20,000 particles, per-particle E, 200 substeps at dt 1e-4, checkpoints every 20."""
    from oracle import bridge, cref
    from oracle import mpm_adjoint as AD

    d = W.diff_elastic()
    loss, gv, gE = _grads(d, checkpoint_every=20)
    p, mats, st = bridge.from_desc(d, np.float64)
    n = d.n_particles
    tgt = d.meta["target"]
    v0 = d.meta["v0"]
    E = d.E_particle

    def L(v, Ev):
        s = dict(st)
        s["v"] = np.tile(v, (n, 1))
        mu, lam = AD.lame_of_E(Ev, 0.3)
        out, rc = cref.substeps(p, mats, s, d.n_substeps, mu_p=mu, lam_p=lam)
        assert rc == 0
        return float(((out["x"].mean(0) - tgt) ** 2).sum())

    h = 1e-4
    for c in range(3):
        e = np.zeros(3)
        e[c] = h
        fd = (L(v0 + e, E) - L(v0 - e, E)) / (2 * h)
        print(f"\n[accuracy] grad v0[{c}]: adjoint {gv[c]:.6e}  fp64 FD {fd:.6e}  rel {abs(gv[c] - fd) / abs(fd):.2e}")
        assert abs(gv[c] - fd) <= 2e-2 * max(abs(fd), 1e-3 * np.abs(gv).max()), (c, gv[c], fd)
    k = int(np.argmax(np.abs(gE)))
    hE = 1e-4 * E[k]
    Ep, Em = E.copy(), E.copy()
    Ep[k] += hE
    Em[k] -= hE
    fd = (L(v0, Ep) - L(v0, Em)) / (2 * hE)
    print(f"\n[accuracy] grad E[{k}]: adjoint {gE[k]:.6e}  fp64 FD {fd:.6e}  rel {abs(gE[k] - fd) / abs(fd):.2e}")
    assert abs(gE[k] - fd) <= 5e-2 * abs(fd), (gE[k], fd)


def _fd_setup(d, actu=None, mdir=None):
    from oracle import bridge, cref
    from oracle import mpm_adjoint as AD

    p, mats, st = bridge.from_desc(d, np.float64)
    n = d.n_particles
    tgt = d.meta["target"]

    def L(v, Ev, a=None):
        s = dict(st)
        s["v"] = np.tile(v, (n, 1))
        if a is not None:
            s["actu"] = a
            s["mdir"] = mdir
        mu, lam = AD.lame_of_E(Ev, 0.3)
        out, rc = cref.substeps(p, mats, s, d.n_substeps, mu_p=mu, lam_p=lam)
        assert rc == 0
        return float(((out["x"].mean(0) - tgt) ** 2).sum())

    return L


def test_neo_hookean_adjoint_against_fp64_finite_differences():
    d = W.diff_elastic(n=2000, n_substeps=120)
    d.materials = [("elastic", dict(E=1e5, nu=0.3, rho=1000.0, model="neohooken"))]
    loss, gv, gE = _grads(d, checkpoint_every=20)
    L = _fd_setup(d)
    v0, E = d.meta["v0"], d.E_particle
    h = 1e-4
    for c in (0, 2):
        e = np.zeros(3)
        e[c] = h
        fd = (L(v0 + e, E) - L(v0 - e, E)) / (2 * h)
        print(f"\n[accuracy] neo-Hookean grad v0[{c}]: adjoint {gv[c]:.6e}  fp64 FD {fd:.6e}")
        assert abs(gv[c] - fd) <= 2e-2 * max(abs(fd), 1e-3 * np.abs(gv).max()), (c, gv[c], fd)
    k = int(np.argmax(np.abs(gE)))
    hE = 1e-4 * E[k]
    Ep, Em = E.copy(), E.copy()
    Ep[k] += hE
    Em[k] -= hE
    fd = (L(v0, Ep) - L(v0, Em)) / (2 * hE)
    print(f"\n[accuracy] neo-Hookean grad E[{k}]: adjoint {gE[k]:.6e}  fp64 FD {fd:.6e}")
    assert abs(gE[k] - fd) <= 5e-2 * abs(fd), (gE[k], fd)


def test_muscle_actuation_adjoint_against_fp64_finite_differences():
    """Muscle (neo-Hookean) block with two actuation groups along different fibres:
    dL/d(group actuation) = sum of the per-particle actuation adjoints of the group."""
    from genesis_b200.grad import DifferentiableRollout, rollout

    d = W.diff_elastic(n=2000, n_substeps=120)
    d.materials = [("muscle", dict(E=1e5, nu=0.3, rho=1000.0))]
    n = d.n_particles
    group = (d.pos[:, 0] > np.median(d.pos[:, 0])).astype(np.int64)
    mdir = np.where(group[:, None] == 0, [0.0, 0.0, 1.0], [0.0, 0.6, 0.8])
    d.meta["muscle_dir"] = mdir
    a_grp = np.array([0.3, -0.2])
    sim = DifferentiableRollout(d, checkpoint_every=20)
    v0 = torch.tensor(d.meta["v0"], dtype=torch.float32, device="cuda")
    E = torch.tensor(d.E_particle, dtype=torch.float32, device="cuda")
    a = torch.tensor(a_grp[group], dtype=torch.float32, device="cuda", requires_grad=True)
    x = rollout(v0, E, sim, actu=a)
    tgt = torch.tensor(d.meta["target"], dtype=torch.float32, device="cuda")
    ((x.mean(0) - tgt) ** 2).sum().backward()
    ga = a.grad.cpu().numpy().astype(np.float64)
    g_grp = np.array([ga[group == 0].sum(), ga[group == 1].sum()])
    L = _fd_setup(d, mdir=mdir)
    h = 1e-3
    for gi in range(2):
        ap, am = a_grp.copy(), a_grp.copy()
        ap[gi] += h
        am[gi] -= h
        fd = (L(d.meta["v0"], d.E_particle, ap[group]) - L(d.meta["v0"], d.E_particle, am[group])) / (2 * h)
        print(f"\n[accuracy] muscle grad actu[group {gi}]: adjoint {g_grp[gi]:.6e}  fp64 FD {fd:.6e}")
        assert abs(g_grp[gi] - fd) <= 3e-2 * max(abs(fd), 1e-3 * np.abs(g_grp).max()), (gi, g_grp[gi], fd)
    assert n == 2000


def test_position_and_per_particle_velocity_gradients_against_fp64_fd():
    """dL/d(position offset) (entity.set_position) and per-particle dL/dv0 from the adjoint,
    against float64 central differences of the C restatement (particle_entity.py:415-481)."""
    from oracle import bridge, cref
    from oracle import mpm_adjoint as AD

    from genesis_b200.grad import DifferentiableRollout, rollout

    d = W.diff_elastic(n=2000, n_substeps=80)
    sim = DifferentiableRollout(d, checkpoint_every=20)
    n = d.n_particles
    v0 = torch.tensor(np.tile(d.meta["v0"], (n, 1)), dtype=torch.float32, device="cuda", requires_grad=True)
    off = torch.zeros(3, dtype=torch.float32, device="cuda", requires_grad=True)
    E = torch.tensor(d.E_particle, dtype=torch.float32, device="cuda")
    tgt = torch.tensor(d.meta["target"], dtype=torch.float32, device="cuda")
    x = rollout(v0, E, sim, x0=off)
    ((x.mean(0) - tgt) ** 2).sum().backward()
    g_off = off.grad.cpu().numpy().astype(np.float64)
    g_v = v0.grad.cpu().numpy().astype(np.float64)
    assert g_v.shape == (n, 3)

    p, mats, st = bridge.from_desc(d, np.float64)
    mu, lam = AD.lame_of_E(d.E_particle, 0.3)

    def L(dx=np.zeros(3), dv=None):
        s = dict(st)
        s["x"] = st["x"] + dx
        v = np.tile(d.meta["v0"], (n, 1))
        if dv is not None:
            v = v + dv
        s["v"] = v
        out, rc = cref.substeps(p, mats, s, d.n_substeps, mu_p=mu, lam_p=lam)
        assert rc == 0
        return float(((out["x"].mean(0) - d.meta["target"]) ** 2).sum())

    h = 1e-5
    for c in range(3):
        e = np.zeros(3)
        e[c] = h
        fd = (L(dx=e) - L(dx=-e)) / (2 * h)
        print(f"\n[accuracy] grad position offset[{c}]: adjoint {g_off[c]:.6e}  fp64 FD {fd:.6e}")
        assert abs(g_off[c] - fd) <= 2e-2 * max(abs(fd), 1e-3 * np.abs(g_off).max()), (c, g_off[c], fd)
    k = int(np.argmax(np.abs(g_v[:, 2])))
    dv = np.zeros((n, 3))
    dv[k, 2] = 1e-3
    fd = (L(dv=dv) - L(dv=-dv)) / 2e-3
    print(f"\n[accuracy] grad v0[particle {k}, z]: adjoint {g_v[k, 2]:.6e}  fp64 FD {fd:.6e}")
    assert abs(g_v[k, 2] - fd) <= 5e-2 * abs(fd), (g_v[k, 2], fd)


def test_trajectory_loss_gradient_against_fp64_fd():
    """A loss over the positions after every 20 substeps (the reference's scripts sum a loss
    over get_state() each step): the recorded states' gradients enter the adjoint at their
    substeps; dL/dv0 and dL/dE against float64 central differences."""
    from oracle import bridge, cref
    from oracle import mpm_adjoint as AD

    from genesis_b200.grad import DifferentiableRollout, rollout

    d = W.diff_elastic(n=2000, n_substeps=80)
    sim = DifferentiableRollout(d, checkpoint_every=30)  # record points fall inside segments
    rec = [0, 20, 40, 60, 80]
    v0 = torch.tensor(d.meta["v0"], dtype=torch.float32, device="cuda", requires_grad=True)
    E = torch.tensor(d.E_particle, dtype=torch.float32, device="cuda", requires_grad=True)
    tgt = torch.tensor(d.meta["target"], dtype=torch.float32, device="cuda")
    xs = rollout(v0, E, sim, record=rec)
    assert xs.shape == (len(rec), d.n_particles, 3)
    ((xs.mean(1) - tgt) ** 2).sum().backward()
    gv, gE = v0.grad.cpu().numpy().astype(np.float64), E.grad.cpu().numpy().astype(np.float64)
    final = rollout(v0.detach(), E.detach(), sim)
    # splitting the substep calls changes nothing but the order of the grid's float atomics
    assert torch.allclose(xs[-1], final, atol=1e-6)
    stale = rollout(v0, E, sim, record=rec)
    rollout(v0.detach(), E.detach(), sim)  # a later forward replaces the checkpoints
    with pytest.raises(Exception, match="backward before the next forward"):
        stale.sum().backward()

    p, mats, st = bridge.from_desc(d, np.float64)
    n = d.n_particles

    def L(v, Ev):
        s = dict(st)
        s["v"] = np.tile(v, (n, 1))
        mu, lam = AD.lame_of_E(Ev, 0.3)
        loss = float(((s["x"].mean(0) - d.meta["target"]) ** 2).sum())
        for _ in range(4):
            s, rc = cref.substeps(p, mats, s, 20, mu_p=mu, lam_p=lam)
            assert rc == 0
            loss += float(((s["x"].mean(0) - d.meta["target"]) ** 2).sum())
        return loss

    h = 1e-4
    for c in range(3):
        e = np.zeros(3)
        e[c] = h
        fd = (L(d.meta["v0"] + e, d.E_particle) - L(d.meta["v0"] - e, d.E_particle)) / (2 * h)
        print(f"\n[accuracy] trajectory grad v0[{c}]: adjoint {gv[c]:.6e}  fp64 FD {fd:.6e}")
        assert abs(gv[c] - fd) <= 2e-2 * max(abs(fd), 1e-3 * np.abs(gv).max()), (c, gv[c], fd)
    k = int(np.argmax(np.abs(gE)))
    Ep, Em = d.E_particle.copy(), d.E_particle.copy()
    Ep[k] *= 1 + 1e-4
    Em[k] *= 1 - 1e-4
    fd = (L(d.meta["v0"], Ep) - L(d.meta["v0"], Em)) / (2e-4 * d.E_particle[k])
    print(f"\n[accuracy] trajectory grad E[{k}]: adjoint {gE[k]:.6e}  fp64 FD {fd:.6e}")
    assert abs(gE[k] - fd) <= 5e-2 * abs(fd), (gE[k], fd)
