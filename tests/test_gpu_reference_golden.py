"""The CUDA path against fixtures made by running the REFERENCE's own MPM code
(tests/golden/ref_*.npz, from make_reference_golden.py: Genesis's mpm_solver.py,
legacy_coupler.py, boundaries.py and materials/MPM/*.py executed unchanged on a numpy
stand-in for gstaichi, float64).

* every material variant's return mapping (F_new, Jp_new) and stress (the precision-32
  model's fixture, ref_functions_m32), read back after one p2g from particles whose stencils
  do not overlap (so each grid node's momentum is one particle's stress contribution);
* whole substeps over 9 material variants (random F, C, Jp, velocity; inactive particles;
  muscle actuation) and a cube thrown at the floor: grid mass/momentum after the first p2g
  and the full state after each snapshot.

The whole-substep fixtures exist twice: the reference's precision-64 run, and its
precision-32 model computed in float64 (float32 gs.EPS, "_m32").  The float32 CUDA path is
held to the precision-32 model; its distance from the precision-64 run is printed (-s).

Tolerances (float32 kernels against the float64 fixtures): positions 1e-5 of the 1 m domain
after every snapshot; F and Jp 1e-5, or 4x the float32 C restatement's own deviation from the
same fixture plus 1e-6 where that is larger (after 20 substeps of the random mixed scene's
plastic flow, float32 itself deviates by ~5e-6 in F and Jp); velocities no more than 4x the
float32 C restatement's own deviation, plus 1e-6 m/s (velocities reach 1.7 m/s with |C| up to
70 /s in the random mixed scene, where float32 itself deviates by ~1e-5 m/s); grid mass and
momentum totals 1e-6 relative, per node 1e-5 of the largest node; F_new 2e-6 and Jp_new 2e-6
relative to the largest entry of each variant; stress (through the momentum it scatters) 1e-5
of each particle's largest node value, or 4x the float32 C restatement's own stress error where
that is larger (a yielding von Mises particle's stress hangs on s_new - 1 ~ 1e-2, which a
float32 SVD's singular values leave ~1e-5 uncertain), plus the shared tile's fixed-point
resolution, 2^-22 of the chunk's payload bound per contribution (asserted at 2^-21).
"""

import json
import os

import numpy as np
import pytest
import torch

from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(__file__), "golden")


def _dense(rt):
    from genesis_b200.engine.runtime import block_major_to_dense

    mm, _ = rt.grid_views()
    torch.cuda.synchronize()
    return block_major_to_dense(mm.cpu().numpy().astype(np.float64), rt.specs[0], int(rt._insts[0].blk_base))


def _weights(fx):
    return [0.5 * (1.5 - fx) ** 2, 0.75 - (fx - 1.0) ** 2, 0.5 * (fx - 0.5) ** 2]


def test_material_functions_and_stress_match_reference():
    from genesis_b200.engine.runtime import runtime_from_descs

    z = np.load(os.path.join(HERE, "ref_functions_m32.npz"))  # the precision-32 model, as the kernels
    meta = json.loads(str(z["meta"]))
    variants = meta["variants"]
    nv, n = len(variants), len(z["m0_F_tmp"])
    density, psize, dt = 96, 0.01, 1e-4
    dx = 1.0 / density
    # isolated particles: bases 6 cells apart, so no two stencils share a node and no two
    # particles share a 4^3 grid block (each chunk's fixed-point scale is its one particle's)
    ks = np.stack(np.meshgrid(*[np.arange(1, 16)] * 3, indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.default_rng(3)
    sel = rng.permutation(len(ks))[: nv * n]
    pos = (6 * ks[sel] + 1.0) * dx + rng.uniform(-0.2 * dx, 0.2 * dx, size=(nv * n, 3))
    mat_idx = np.repeat(np.arange(nv), n)
    d = W.SceneDesc(name="ref_functions", grid_density=density, particle_size=psize, dt=dt, n_substeps=1, pos=pos,
                    vel=np.zeros((nv * n, 3)), mat_idx=mat_idx, materials=[(k, dict(kw)) for k, kw in variants],
                    gravity=(0.0, 0.0, 0.0))
    rt = runtime_from_descs([d], use_graphs=False)
    F0 = np.concatenate([z[f"m{v}_F_tmp"] for v in range(nv)])
    Jp0 = np.concatenate([z[f"m{v}_Jp"] for v in range(nv)])
    rt.set_state(pos=pos, C_=np.zeros((nv * n, 3, 3)), F=F0, Jp=Jp0)
    mus = [v for v, (k, _) in enumerate(variants) if k == "muscle"]
    for v in mus:
        idx = np.arange(v * n, (v + 1) * n)
        rt.set_muscle_group(idx, np.zeros(n, dtype=np.int64))
        rt.set_actu_by_group(idx, z[f"m{v}_actu"][:, None])
        rt.set_muscle_direction(idx, z[f"m{v}_mdir"])
    rt.sort()
    rt.p2g()
    st = rt.get_state(("F", "Jp"))
    torch.cuda.synchronize()
    F = st["F"].cpu().numpy().astype(np.float64)
    Jp = st["Jp"].cpu().numpy().astype(np.float64)
    grid = _dense(rt)
    lo = np.round(density * np.asarray(d.lower_bound)).astype(int)
    scale = -dt * (psize**3 * 1e3) * 4 * density * density
    # the float32 C restatement on the same isolated particles: after one substep an isolated
    # particle's C is A / m = scale * stress / m (the B-spline's moments), so its stress is
    # read back as C m / scale; its deviation from the fixture is float32's own, with its own
    # float32 SVD (near a yield surface the stress depends on s_new - 1 ~ 1e-2, so the SVD's
    # few-ulp singular values already cost ~1e-5 of it)
    from oracle import cref
    from oracle import mpm_ref as R

    p32 = R.Params(grid_density=density, particle_size=psize, dt=dt, gravity=(0.0, 0.0, 0.0), dtype=np.float32)
    p32.eps = float(np.finfo(np.float32).eps)
    mats32 = [R.make_material(k, **dict(kw)) for k, kw in variants]
    st32 = R.make_state(pos, mats32, mat_idx, np.float32)
    st32.update(F=F0.astype(np.float32), Jp=Jp0.astype(np.float32))
    if mus:
        actu32 = np.zeros(nv * n, np.float32)
        mdir32 = np.tile(np.float32([0, 0, 1]), (nv * n, 1))
        for v in mus:
            actu32[v * n:(v + 1) * n] = z[f"m{v}_actu"]
            mdir32[v * n:(v + 1) * n] = z[f"m{v}_mdir"]
        st32.update(actu=actu32, mdir=mdir32)
    out32, rc32 = cref.substeps(p32, mats32, st32, 1)
    assert rc32 == 0
    mass = np.array([R.particle_mass(p32, mats32[k]) for k in mat_idx])
    stress32 = out32["C"].astype(np.float64) * (mass / scale)[:, None, None]
    for v in range(nv):
        sl = slice(v * n, (v + 1) * n)
        want_F, want_Jp, want_s = z[f"m{v}_F_new"], z[f"m{v}_Jp_new"], z[f"m{v}_stress"]
        eF = np.abs(F[sl] - want_F).max() / max(1.0, np.abs(want_F).max())
        eJ = np.abs(Jp[sl] - want_Jp).max() / max(1.0, np.abs(want_Jp).max())
        assert eF < 2e-6 and eJ < 2e-6, (variants[v], eF, eJ)
        # stress: node momentum = w * (scale * stress) @ dpos (v = 0, C = 0)
        xi = pos[sl] * density
        base = np.floor(xi - 0.5).astype(int)
        fx = xi - base
        w = _weights(fx)
        got, want = [], []
        for i in range(3):
            for j in range(3):
                for k in range(3):
                    off = np.array([i, j, k])
                    wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
                    dpos = (off - fx) * dx
                    want.append(wt[:, None] * np.einsum("nab,nb->na", scale * want_s, dpos))
                    node = base + off - lo
                    got.append(grid[node[:, 0], node[:, 1], node[:, 2], :3])
        got, want = np.stack(got), np.stack(want)  # [27, n, 3]
        # the tile's payload bound of each particle (v = 0, C = 0): 1.5 dx max_i sum_j |A_ij|
        bound = 1.5 * dx * np.abs(scale * want_s).sum(axis=2).max(axis=1)
        err = np.abs(got - want).max(axis=(0, 2))
        # float32's own deviation, in node-momentum units (w <= 1, |dpos| <= 1.5 dx per axis)
        e32 = 1.5 * dx * np.abs(scale * (stress32[sl] - want_s)).sum(axis=2).max(axis=1)
        tol = np.maximum(1e-5 * np.abs(want).max(axis=(0, 2)), 4 * e32) + 2.0**-21 * bound
        print(f"\n[reference] {variants[v][0]} {variants[v][1]}: F_new {eF:.1e}, Jp_new {eJ:.1e}, stress "
              f"max err / tol {float((err / tol).max()):.2f} (float32 C restatement: max rel. stress err "
              f"{float((np.abs(stress32[sl] - want_s).max(axis=(1, 2)) / np.abs(want_s).max(axis=(1, 2))).max()):.1e})")
        assert (err <= tol).all(), (variants[v], float((err / tol).max()))


def _f32_oracle(z, meta, n):
    """The float32 C restatement from the fixture's inputs, n substeps (same model)."""
    from oracle import cref
    from oracle import mpm_ref as R

    p = R.Params(grid_density=meta["grid_density"], lower_bound=tuple(meta["lower_bound"]),
                 upper_bound=tuple(meta["upper_bound"]), particle_size=meta["particle_size"], dt=meta["dt"],
                 gravity=tuple(meta["gravity"]), dtype=np.float32)
    mats = [R.make_material(k, **dict(kw)) for k, kw in meta["materials"]]
    st = R.make_state(z["pos"], mats, z["mat_idx"], np.float32, v=z["vel"], active=z["active"])
    st.update(C=z["C"].astype(np.float32), F=z["F"].astype(np.float32), Jp=z["Jp"].astype(np.float32))
    if "muscle_idx" in z.files:
        k = len(z["pos"])
        actu = np.zeros(k, np.float32)
        mdir = np.tile(np.float32([0, 0, 1]), (k, 1))
        actu[z["muscle_idx"]] = z["muscle_actu"][z["muscle_group"]]
        mdir[z["muscle_idx"]] = z["muscle_dir"]
        st.update(actu=actu, mdir=mdir)
    out, rc = cref.substeps(p, mats, st, n)
    assert rc == 0
    return out


def _scene(name):
    from genesis_b200.engine.runtime import runtime_from_descs

    z = np.load(os.path.join(HERE, f"{name}.npz"))
    meta = json.loads(str(z["meta"]))
    d = W.SceneDesc(name=name, grid_density=meta["grid_density"], particle_size=meta["particle_size"], dt=meta["dt"],
                    n_substeps=meta["snapshots"][-1], pos=z["pos"], vel=z["vel"], mat_idx=z["mat_idx"],
                    materials=[(k, dict(kw)) for k, kw in meta["materials"]],
                    lower_bound=tuple(meta["lower_bound"]), upper_bound=tuple(meta["upper_bound"]),
                    gravity=tuple(meta["gravity"]))
    rt = runtime_from_descs([d], sort_interval=4)
    rt.set_state(pos=z["pos"], vel=z["vel"], C_=z["C"], F=z["F"], Jp=z["Jp"], active=z["active"].astype(np.uint8))
    if "muscle_idx" in z.files:
        idx = z["muscle_idx"]
        rt.set_muscle_group(idx, z["muscle_group"])
        rt.set_actu_by_group(idx, np.tile(z["muscle_actu"], (len(idx), 1)))
        rt.set_muscle_direction(idx, z["muscle_dir"])
    return z, meta, rt


@pytest.mark.parametrize("name", ["ref_mixed_m32", "ref_cube_m32"])
def test_first_p2g_grid_matches_reference(name):
    z, meta, rt = _scene(name)
    rt.sort()
    rt.p2g()
    g = _dense(rt)
    gm, gp = z["grid_mass"], z["grid_mom"]
    assert abs(g[..., 3].sum() - gm.sum()) <= 1e-6 * gm.sum()
    mscale = np.abs(gp).sum()
    assert np.abs(g[..., :3].reshape(-1, 3).sum(0) - gp.reshape(-1, 3).sum(0)).max() <= 1e-6 * mscale
    assert np.abs(g[..., 3] - gm).max() <= 1e-5 * gm.max()
    assert np.abs(g[..., :3] - gp).max() <= 1e-5 * np.abs(gp).max()


@pytest.mark.parametrize("name", ["ref_mixed", "ref_cube"])
def test_substeps_match_reference(name):
    z, meta, rt = _scene(name + "_m32")
    z64 = np.load(os.path.join(HERE, f"{name}.npz"))
    done = 0
    act = z["active"]
    for n in meta["snapshots"]:
        rt.substeps(n - done)
        done = n
        st = rt.get_state()
        torch.cuda.synchronize()
        got = {k: st[k].cpu().numpy().astype(np.float64) for k in ("pos", "vel", "F", "Jp")}
        ex = np.abs(got["pos"] - z[f"x_{n}"]).max()
        ev = np.abs(got["vel"] - z[f"v_{n}"]).max()
        eF = np.abs(got["F"] - z[f"F_{n}"]).max()
        eJ = np.abs(got["Jp"] - z[f"Jp_{n}"]).max()
        o32 = _f32_oracle(z, meta, n)
        e32v = np.abs(o32["v"] - z[f"v_{n}"]).max()
        e32F = np.abs(o32["F"] - z[f"F_{n}"]).max()
        e32J = np.abs(o32["Jp"] - z[f"Jp_{n}"]).max()
        ex64 = np.abs(got["pos"] - z64[f"x_{n}"]).max()
        ev64 = np.abs(got["vel"] - z64[f"v_{n}"]).max()
        print(f"\n[reference] {name} after {n}: precision-32 model |dx| {ex:.2e} |dv| {ev:.2e} (float32 C "
              f"restatement {e32v:.2e}) |dF| {eF:.2e} ({e32F:.2e}) |dJp| {eJ:.2e} ({e32J:.2e}); precision 64 "
              f"|dx| {ex64:.2e} |dv| {ev64:.2e}")
        assert ex < 1e-5, (n, ex)
        assert eF <= max(1e-5, 4 * e32F + 1e-6) and eJ <= max(1e-5, 4 * e32J + 1e-6), (n, eF, e32F, eJ, e32J)
        assert ev <= 4 * e32v + 1e-6, (n, ev, e32v)
        assert np.array_equal(got["pos"][~act], z["pos"][~act].astype(np.float32).astype(np.float64))
    assert rt.status() == 0
