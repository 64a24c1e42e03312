"""Generate golden fixtures by running the REFERENCE's own MPM code (not the oracle).

    python tests/golden/make_reference_golden.py [path-to-Genesis-checkout]
        (default: $GENESIS_REFERENCE, else /root/reference)

The reference's files are imported unchanged from the checkout with ``ti_numpy`` standing
in for gstaichi (see that module for what is emulated; the one substitution is ti.svd, a
compiled routine whose source is absent, replaced by LAPACK in ti.svd's convention).  All
runs are float64 (the reference's ``precision="64"``).  Written here:

  ref_functions.npz    per material variant, 96 deformation gradients F_tmp (singular values
                       0.3-1.6, some nearly repeated) through the reference's update_F_S_Jp and
                       update_stress (materials/MPM/*.py, J = det S as mpm_solver.py:305 takes
                       it); CubeBoundary.impose_pos_vel (boundaries.py:23-33) on 96 points at
                       and beyond the walls; backward_svd (mpm_solver.py:1112-1129) on 96
                       random (grad_U, grad_S, grad_V) at random F.
  ref_mixed.npz        216 particles of 9 material variants (Elastic corotated / neo-Hookean,
                       Muscle with 2 actuation groups, ElastoPlastic von Mises / clamp, Liquid
                       inviscid / viscous, Sand, Snow) with random F, C, Jp and velocity, a sixth
                       of them inactive, stepped by MPMSolver + LegacyCoupler's kernels: grid
                       mass/momentum after the first p2g, full state after 1, 5 and 20 substeps.
  ref_cube.npz         an Elastic cube (E 1e5, nu 0.3, rho 1000: the 32,768-particle benchmark
                       cube's material) of 216 jittered lattice particles thrown at the floor of
                       a 64-per-metre grid, dt 1e-4: state after 1, 20 and 60 substeps.
  ref_force_fields.npz the reference's force fields (engine/force_fields.py: Constant, Wind,
                       Point, Drag, Vortex, Turbulence seeded and unseeded) through their own
                       get_acc at 96 random positions and velocities each, and a scene of two
                       blocks (Elastic, Liquid) under Constant + Vortex + Turbulence + Drag +
                       Point + Wind stepped by MPMSolver + LegacyCoupler (the fields enter
                       mpm_grid_op, legacy_coupler.py:377-379): state after 1, 5 and 15
                       substeps, precision-32 model.
  ref_functions_m32.npz, ref_mixed_m32.npz, ref_cube_m32.npz
                       the same with the reference's precision-32 model in float64
                       arithmetic: gs.EPS = float32 epsilon (genesis/__init__.py:205-206, the
                       grid-mass threshold and the eps of Matrix.norm in the plastic return
                       mappings), everything else float64.  A float32 run of the reference
                       computes this model; the float32 CUDA path is held to it.

Only this script reads the reference checkout; the tests read the committed .npz files.
"""

from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

import ti_numpy as T  # noqa: E402

# (kind, kwargs) as genesis_b200.workloads / oracle.mpm_ref.make_material take them
VARIANTS = [
    ("elastic", dict(E=1e5, nu=0.3)),
    ("elastic", dict(E=2e5, nu=0.25, model="neohooken")),
    ("muscle", dict(E=1e5, nu=0.3)),
    ("elastoplastic", dict(E=1e5, nu=0.3, von_mises_yield_stress=1e3)),
    ("elastoplastic", dict(E=1e5, nu=0.3, use_von_mises=False)),
    ("liquid", dict(E=1e5, nu=0.2)),
    ("liquid", dict(E=1e5, nu=0.2, viscous=True)),
    ("sand", dict(friction_angle=40)),
    ("snow", dict(yield_lower=2.5e-2, yield_higher=7.5e-3)),
]


def ref_material(ref, kind, kw):
    kw = dict(kw)
    cls = dict(elastic=ref.Elastic, elastoplastic=ref.ElastoPlastic, liquid=ref.Liquid, sand=ref.Sand,
               snow=ref.Snow, muscle=ref.Muscle)[kind]
    if kind != "sand" and kind != "snow":
        kw.setdefault("sampler", "random")
    return cls(**kw)


def rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1),
    ], -2)


def random_F(rng, n):
    """F = R1 diag(s) R2^T with s in [0.3, 1.6]; every fourth sample has two singular values
    within 1e-3 of each other, every eighth is a mild strain (s in [0.97, 1.03])."""
    s = rng.uniform(0.3, 1.6, size=(n, 3))
    s[::4, 1] = s[::4, 0] * (1 + rng.uniform(-1e-3, 1e-3, size=s[::4, 0].shape))
    s[1::8] = rng.uniform(0.97, 1.03, size=s[1::8].shape)
    return rotations(rng, n) @ (s[:, :, None] * np.swapaxes(rotations(rng, n), 1, 2))


def functions_fixture(ref, seed=20):
    rng = np.random.default_rng(seed)
    n = 96
    out = {}
    for vi, (kind, kw) in enumerate(VARIANTS):
        m = ref_material(ref, kind, kw)
        F = random_F(rng, n)
        if kind == "sand":
            Jp = rng.uniform(-0.3, 0.3, n)
        elif kind == "snow":
            Jp = rng.uniform(0.7, 1.3, n)
        else:
            Jp = np.ones(n)
        actu = rng.uniform(-0.5, 0.5, n)
        mdir = rng.normal(size=(n, 3))
        mdir /= np.linalg.norm(mdir, axis=1, keepdims=True)
        Fn, Sn, Jn, st = np.zeros((n, 3, 3)), np.zeros((n, 3, 3)), np.zeros(n), np.zeros((n, 3, 3))
        for i in range(n):
            U, S, V = T.svd(F[i])
            J = S.determinant()
            f_new, s_new, jp_new = m.update_F_S_Jp(J=J, F_tmp=np.asarray(F[i]).view(T.TiArr),
                                                   U=U, S=S, V=V, Jp=Jp[i])
            stress = m.update_stress(U=U, S=s_new, V=V, F_tmp=np.asarray(F[i]).view(T.TiArr), F_new=f_new, J=J,
                                     Jp=Jp[i], actu=actu[i], m_dir=np.asarray(mdir[i]).view(T.TiArr))
            Fn[i], Sn[i], Jn[i], st[i] = f_new, s_new, jp_new, stress
        out[f"m{vi}_F_tmp"] = F
        out[f"m{vi}_Jp"] = Jp
        out[f"m{vi}_actu"] = actu
        out[f"m{vi}_mdir"] = mdir
        out[f"m{vi}_F_new"] = Fn
        out[f"m{vi}_S_new"] = Sn
        out[f"m{vi}_Jp_new"] = Jn
        out[f"m{vi}_stress"] = st
    # CubeBoundary on the benchmark domain's padded box
    lo, hi = np.full(3, 3 / 64), np.full(3, 1 - 3 / 64)
    b = ref.CubeBoundary(lower=lo, upper=hi)
    pos = rng.uniform(-0.05, 1.05, size=(n, 3))
    pos[::3] = np.where(rng.random((len(pos[::3]), 3)) < 0.5, lo, hi)  # exactly on a wall
    vel = rng.normal(size=(n, 3))
    vel[::5, 0] = 0.0
    bp, bv = np.zeros((n, 3)), np.zeros((n, 3))
    for i in range(n):
        p_, v_ = b.impose_pos_vel(np.asarray(pos[i]).view(T.TiArr), np.asarray(vel[i]).view(T.TiArr))
        bp[i], bv[i] = p_, v_
    out.update(bnd_lo=lo, bnd_hi=hi, bnd_pos=pos, bnd_vel=vel, bnd_pos_out=bp, bnd_vel_out=bv)
    # backward_svd at random F
    F = random_F(rng, n)
    gU, gS, gV = rng.normal(size=(3, n, 3, 3))
    res = np.zeros((n, 3, 3))
    Us, Ss, Vs = np.zeros((n, 3, 3)), np.zeros((n, 3, 3)), np.zeros((n, 3, 3))
    for i in range(n):
        U, S, V = T.svd(F[i])
        Us[i], Ss[i], Vs[i] = U, S, V
        res[i] = ref.backward_svd(*(np.asarray(x).view(T.TiArr) for x in (gU[i], gS[i], gV[i])), U, S, V)
    out.update(bsvd_U=Us, bsvd_S=Ss, bsvd_V=Vs, bsvd_gU=gU, bsvd_gS=gS, bsvd_gV=gV, bsvd_out=res)
    meta = dict(variants=[[k, kw] for k, kw in VARIANTS], eps=ref.gs.EPS)
    return meta, out


def run_scene(ref, name, blocks_spec, grid_density, upper, particle_size, dt, gravity, state, snapshots,
              muscle=None):
    blocks = [(ref_material(ref, k, kw), pos) for (k, kw), pos in blocks_spec]
    sc = T.Scene(ref, grid_density, (0.0, 0.0, 0.0), upper, particle_size, dt, gravity, blocks)
    sc.set_state(**state)
    if muscle is not None:
        sc.solver.particles.member("actu")[0, :, 0] = muscle["actu"]
        sc.solver.particles_info.member("muscle_direction")[:] = muscle["dir"]
    rec = {}
    done = 0
    t0 = time.time()
    for n in snapshots:
        while done < n:
            gm, gp = sc.substep()
            if done == 0:
                rec["grid_mass"], rec["grid_mom"] = gm, gp
            done += 1
        s = sc.state()
        for k, kk in (("x", "pos"), ("v", "vel"), ("C", "C"), ("F", "F"), ("Jp", "Jp")):
            rec[f"{k}_{n}"] = s[kk]
    print(f"{name}: {sum(p.shape[0] for _, p in blocks_spec)} particles, {snapshots[-1]} substeps, "
          f"{time.time() - t0:.1f} s")
    return rec


def mixed_fixture(ref, seed=21):
    rng = np.random.default_rng(seed)
    n_per = 24
    upper = (0.5, 0.5, 0.5)
    specs, pos_all, mat_idx = [], [], []
    for vi, spec in enumerate(VARIANTS):
        pos = rng.uniform(0.12, 0.38, size=(n_per, 3))
        specs.append((spec, pos))
        pos_all.append(pos)
        mat_idx += [vi] * n_per
    pos = np.concatenate(pos_all)
    N = pos.shape[0]
    mat_idx = np.array(mat_idx)
    kinds = np.array([VARIANTS[i][0] for i in mat_idx])
    vel = rng.normal(0.0, 0.5, size=(N, 3))
    C = rng.normal(0.0, 4.0, size=(N, 3, 3))
    F = np.eye(3) + rng.normal(0.0, 0.04, size=(N, 3, 3))
    Jp = np.where(kinds == "sand", rng.uniform(-0.03, 0.03, N), np.where(kinds == "snow", rng.uniform(0.9, 1.1, N), 1.0))
    active = (np.arange(N) % 6) != 5
    mus = np.nonzero(kinds == "muscle")[0]
    group = (np.arange(mus.size) % 2).astype(np.int64)
    actu_groups = np.array([0.4, -0.25])
    mdir = rng.normal(size=(mus.size, 3))
    mdir /= np.linalg.norm(mdir, axis=1, keepdims=True)
    actu = np.zeros(N)
    actu[mus] = actu_groups[group]
    dirs = np.tile([0.0, 0.0, 1.0], (N, 1))
    dirs[mus] = mdir
    dt, density, psize, grav = 2e-4, 32, 0.01, (0.0, 0.0, -9.8)
    snaps = [1, 5, 20]
    rec = run_scene(ref, "ref_mixed", specs, density, upper, psize, dt, grav,
                    dict(vel=vel, C=C, F=F, Jp=Jp, active=active), snaps, muscle=dict(actu=actu, dir=dirs))
    meta = dict(name="ref_mixed", grid_density=density, lower_bound=[0.0] * 3, upper_bound=list(upper),
                particle_size=psize, dt=dt, gravity=list(grav), materials=[[k, kw] for k, kw in VARIANTS],
                snapshots=snaps)
    inputs = dict(pos=pos, vel=vel, C=C, F=F, Jp=Jp, active=active, mat_idx=mat_idx, muscle_idx=mus,
                  muscle_group=group, muscle_actu=actu_groups, muscle_dir=mdir)
    return meta, inputs, rec


def cube_fixture(ref, seed=22):
    rng = np.random.default_rng(seed)
    n_side, spacing = 6, 0.1 / 6
    upper = (0.375, 0.375, 0.375)
    dx = 1 / 64
    lower = np.array([0.15, 0.15, 3 * dx + 0.004])
    axes = [lower[d] + (np.arange(n_side) + 0.5) * spacing for d in range(3)]
    pos = np.stack(np.meshgrid(*axes, indexing="ij"), -1).reshape(-1, 3)
    pos = pos + rng.uniform(-0.25 * spacing, 0.25 * spacing, size=pos.shape)
    N = pos.shape[0]
    vel = np.tile([0.3, -0.2, -1.0], (N, 1))
    spec = ("elastic", dict(E=1e5, nu=0.3, rho=1000.0))
    dt, snaps = 1e-4, [1, 20, 60]
    rec = run_scene(ref, "ref_cube", [(spec, pos)], 64, upper, spacing, dt, (0.0, 0.0, -9.8),
                    dict(vel=vel), snaps)
    meta = dict(name="ref_cube", grid_density=64, lower_bound=[0.0] * 3, upper_bound=list(upper),
                particle_size=spacing, dt=dt, gravity=[0.0, 0.0, -9.8], materials=[list(spec)], snapshots=snaps)
    C0 = np.zeros((N, 3, 3))
    F0 = np.broadcast_to(np.eye(3), (N, 3, 3)).copy()
    inputs = dict(pos=pos, vel=vel, C=C0, F=F0, Jp=np.ones(N), active=np.ones(N, bool), mat_idx=np.zeros(N, int))
    return meta, inputs, rec


# (class name, kwargs) of the force-field fixtures; every field is activated
FORCE_FIELDS = [
    ("Constant", dict(direction=(1.0, -2.0, 0.5), strength=2.5)),
    ("Wind", dict(direction=(0.0, 1.0, 0.2), strength=3.0, radius=0.35, center=(0.45, 0.0, 0.5))),
    ("Point", dict(strength=-2.0, position=(0.5, 0.45, 0.55), falloff_pow=1.5, flow=0.3)),
    ("Drag", dict(linear=0.4, quadratic=0.25)),
    ("Vortex", dict(center=(0.42, 0.5, 0.0), strength_perpendicular=5.0, strength_radial=1.0, falloff_pow=2.0,
                    falloff_min=0.05, falloff_max=0.8, damping=0.1)),
    ("Vortex", dict(center=(0.5, 0.5, 0.0))),
    ("Turbulence", dict(strength=2.0, frequency=3, flow=0.1, seed=7)),
    ("Turbulence", dict(strength=1.0, frequency=5)),
]
FIELDS_IN_SCENE = [
    ("Constant", dict(direction=(0.0, 0.0, 1.0), strength=3.0)),
    ("Vortex", dict(center=(0.25, 0.25, 0.0), strength_perpendicular=8.0, strength_radial=2.0, falloff_pow=2.0,
                    falloff_min=0.02, falloff_max=0.4, damping=0.2)),
    ("Turbulence", dict(strength=4.0, frequency=6, flow=0.2, seed=3)),
    ("Drag", dict(linear=0.5, quadratic=0.3)),
    ("Point", dict(strength=1.5, position=(0.3, 0.2, 0.3), falloff_pow=1.0, flow=0.1)),
    ("Wind", dict(direction=(1.0, 0.0, 0.0), strength=2.0, radius=0.05, center=(0.25, 0.25, 0.25))),
]


def force_field_fixture(ref, seed=23):
    ff = T._load("genesis.engine.force_fields", os.path.join(ref.root, "genesis", "engine", "force_fields.py"))
    rng = np.random.default_rng(seed)
    n = 96
    out = {}
    for k, (name, kw) in enumerate(FORCE_FIELDS):
        f = getattr(ff, name)(**kw)
        f.activate()
        pos = rng.uniform(-0.2, 1.2, size=(n, 3))
        vel = rng.normal(0.0, 1.0, size=(n, 3))
        acc = np.stack([np.asarray(f.get_acc(np.asarray(pos[i]).view(T.TiArr), np.asarray(vel[i]).view(T.TiArr),
                                                 0.0, -1)) for i in range(n)])
        out.update({f"f{k}_pos": pos, f"f{k}_vel": vel, f"f{k}_acc": acc})
    # a scene under several fields at once, stepped by the reference's solver and coupler
    specs = [(("elastic", dict(E=2e4, nu=0.3)), rng.uniform(0.18, 0.3, size=(60, 3))),
             (("liquid", dict(E=1e5, nu=0.2)), rng.uniform(0.2, 0.32, size=(60, 3)))]
    blocks = [(ref_material(ref, k, kw), pos) for (k, kw), pos in specs]
    density, upper, psize, dt, grav = 32, (0.5, 0.5, 0.5), 0.01, 5e-4, (0.0, 0.0, -9.8)
    sc = T.Scene(ref, density, (0.0, 0.0, 0.0), upper, psize, dt, grav, blocks)
    N = sum(p.shape[0] for _, p in specs)
    vel = rng.normal(0.0, 0.3, size=(N, 3))
    sc.set_state(vel=vel)
    for name, kw in FIELDS_IN_SCENE:
        f = getattr(ff, name)(**kw)
        f.activate()
        sc.solver._ffs.append(f)
    snaps = [1, 5, 15]
    done = 0
    for s_ in snaps:
        while done < s_:
            sc.substep()
            done += 1
        st = sc.state()
        for a, b in (("x", "pos"), ("v", "vel"), ("F", "F")):
            out[f"scene_{a}_{s_}"] = st[b]
    out["scene_pos"] = np.concatenate([p for _, p in specs])
    out["scene_vel"] = vel
    out["scene_mat_idx"] = np.repeat(np.arange(len(specs)), [p.shape[0] for _, p in specs])
    meta = dict(eps=ref.gs.EPS, fields=[[nm, kw] for nm, kw in FORCE_FIELDS],
                scene=dict(fields=[[nm, kw] for nm, kw in FIELDS_IN_SCENE],
                           materials=[[k, kw] for (k, kw), _ in specs], grid_density=density, upper_bound=list(upper),
                           particle_size=psize, dt=dt, gravity=list(grav), snapshots=snaps))
    return meta, out


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GENESIS_REFERENCE", "/root/reference")
    ref = T.Reference(root, precision="64")
    eps64 = ref.gs.EPS
    for suffix, eps in (("", eps64), ("_m32", float(np.finfo(np.float32).eps))):
        ref.gs.EPS = eps
        meta, out = functions_fixture(ref)
        np.savez_compressed(os.path.join(HERE, f"ref_functions{suffix}.npz"), meta=np.array(json.dumps(meta)), **out)
        print(f"ref_functions{suffix}")
        for fn in (mixed_fixture, cube_fixture):
            meta, inputs, rec = fn(ref)
            meta["eps"] = eps
            meta["name"] += suffix
            np.savez_compressed(os.path.join(HERE, f"{meta['name']}.npz"), meta=np.array(json.dumps(meta)),
                                **inputs, **rec)
    ref.gs.EPS = float(np.finfo(np.float32).eps)
    meta, out = force_field_fixture(ref)
    np.savez_compressed(os.path.join(HERE, "ref_force_fields.npz"), meta=np.array(json.dumps(meta)), **out)
    print("ref_force_fields")
    ref.gs.EPS = eps64


if __name__ == "__main__":
    main()
