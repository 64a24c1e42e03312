"""The CUDA adjoint of every MPM material (mpm_substep_adjoint behind
genesis_b200.grad.rollout) against the float64 restatement of the reference's own backward
(oracle/mpm_adjoint.py: rollout_materials, itself checked against central finite differences
in tests/test_oracle_adjoint_materials.py).

Each scene is a block of particles with per-particle E (log-normal, sigma 0.5) thrown at the
floor, so that it deforms (and yields, for the plastic materials) before the loss
|mean(x_T) - target|^2 is read; the mixed scene holds four blocks (Liquid, Sand, Snow,
ElastoPlastic: the 500k benchmark mix) side by side.  The oracle computes the reference's
precision-32 model (float32 gs.EPS) in float64.  Tolerances: the gradient with respect to the
initial velocity within 2e-3 of its largest component, and the per-particle E gradient within
2e-3 of its largest entry (float32 kernels against a float64 oracle over 40 substeps of plastic
flow).
"""

import numpy as np
import pytest
import torch

from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu

MATERIALS = [
    ("elastic", dict(E=1e5, nu=0.3)),
    ("elastic", dict(E=1e5, nu=0.3, model="neohooken")),
    ("elastoplastic", dict(E=1e5, nu=0.3, von_mises_yield_stress=2e3)),
    ("elastoplastic", dict(E=1e5, nu=0.3, use_von_mises=False)),
    ("liquid", dict(E=1e5, nu=0.2, viscous=True)),
    ("liquid", dict(E=1e5, nu=0.2)),
    ("sand", dict(E=1e5, friction_angle=40)),
    ("snow", dict(E=1e5, yield_lower=2.5e-2, yield_higher=7.5e-3)),
]


def _desc(blocks, seed, T=40):
    """blocks: [(kind, kw, lower corner xy)]; 6^3 particles each, 1.2 mm above the floor's padding."""
    rng = np.random.default_rng(seed)
    density = 32
    dx = 1.0 / density
    spacing = 0.5 * dx
    pos, mat, E = [], [], []
    for mi, (kind, kw, xy) in enumerate(blocks):
        lat = W.jittered_lattice(rng, 6, (xy[0], xy[1], 3 * dx + 0.0012), spacing)
        pos.append(lat)
        mat.append(np.full(len(lat), mi))
        E.append(kw["E"] * np.exp(0.5 * rng.normal(size=len(lat))))
    pos = np.concatenate(pos)
    n = len(pos)
    return W.SceneDesc(name="grad_materials", grid_density=density, particle_size=spacing, dt=2e-4, n_substeps=T,
                       pos=pos, vel=np.zeros((n, 3)), mat_idx=np.concatenate(mat),
                       materials=[(k, dict(kw)) for k, kw, _ in blocks], upper_bound=(0.5, 0.5, 0.5),
                       E_particle=np.concatenate(E))


def _oracle(d, v0, target):
    from oracle import bridge
    from oracle import mpm_adjoint as A

    p, mats, st = bridge.from_desc(d, np.float64, model_dtype=np.float32)
    n = d.n_particles
    st["v"] = np.tile(v0, (n, 1))
    nu = np.array([mats[k].nu for k in d.mat_idx])
    mu = d.E_particle / (2 * (1 + nu))
    lam = d.E_particle * nu / ((1 + nu) * (1 - 2 * nu))
    inviscid = np.array([mats[k].kind == 2 and mats[k].mu == 0.0 for k in d.mat_idx])  # Liquid, not viscous
    mu = np.where(inviscid, 0.0, mu)
    loss, gv0, gmu, glam, _ = A.rollout_materials(p, mats, st, mu, lam, d.n_substeps, target)
    gE = np.where(inviscid, 0.0, gmu / (2 * (1 + nu))) + glam * nu / ((1 + nu) * (1 - 2 * nu))
    return loss, gv0, gE


def _cuda(d, v0, target):
    from genesis_b200.grad import DifferentiableRollout, rollout

    sim = DifferentiableRollout(d, checkpoint_every=10)
    v = torch.tensor(v0, dtype=torch.float32, device="cuda", requires_grad=True)
    E = torch.tensor(d.E_particle, dtype=torch.float32, device="cuda", requires_grad=True)
    tgt = torch.tensor(target, dtype=torch.float32, device="cuda")
    x = rollout(v, E, sim)
    loss = ((x.mean(0) - tgt) ** 2).sum()
    loss.backward()
    assert sim.rt.status() == 0
    return float(loss), v.grad.cpu().numpy().astype(np.float64), E.grad.cpu().numpy().astype(np.float64)


def _check(d, name):
    v0 = np.array([0.4, -0.2, -1.0])
    target = np.array([0.3, 0.2, 0.05])
    lo, go, Eo = _oracle(d, v0, target)
    lc, gc, Ec = _cuda(d, v0, target)
    ev = np.abs(gc - go).max() / np.abs(go).max()
    eE = np.abs(Ec - Eo).max() / np.abs(Eo).max()
    print(f"\n[grad] {name}: loss {lc:.6e} (oracle {lo:.6e}); dL/dv0 rel. err {ev:.1e}; dL/dE rel. err {eE:.1e} "
          f"(max |dL/dE| {np.abs(Eo).max():.2e})")
    assert abs(lc - lo) <= 1e-4 * abs(lo)
    assert ev <= 2e-3, (name, gc, go)
    assert eE <= 2e-3, name


@pytest.mark.parametrize("kind,kw", MATERIALS, ids=lambda x: str(x)[:30])
def test_material_gradient_matches_oracle(kind, kw):
    _check(_desc([(kind, kw, (0.2, 0.2))], seed=4), f"{kind} {kw}")


def test_mixed_scene_gradient_matches_oracle():
    """The benchmark's material mix (Liquid, Sand, Snow, ElastoPlastic with von Mises) in one
    differentiable scene."""
    blocks = [("liquid", dict(E=1e5, nu=0.2), (0.1, 0.1)), ("sand", dict(E=1e5, friction_angle=45), (0.3, 0.1)),
              ("snow", dict(E=1e5, yield_lower=2.5e-2, yield_higher=7.5e-3), (0.1, 0.3)),
              ("elastoplastic", dict(E=1e5, von_mises_yield_stress=1e4), (0.3, 0.3))]
    _check(_desc(blocks, seed=5), "mixed Liquid / Sand / Snow / ElastoPlastic")
