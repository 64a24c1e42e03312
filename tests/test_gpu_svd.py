"""Accuracy of the kernels' 3x3 SVD on ill-conditioned and nearly degenerate F_tmp.

The SVD is not exposed by itself; an ElastoPlastic clamp material whose clamp is wider than
every singular value (yield_lower = 1, yield_higher = 1e6: S_new = S) makes p2g write
F_new = U S V^T, the kernel's reconstruction of F_tmp.  Its error is read in the float64 SVD
basis of F: E = U64^T (F_new - F) V64, so E_ii / s_i is the relative error of singular value
i and E_ij / s_j (i != j) the leak of direction j into i.  Particles are isolated (one per
4^3 block, C = 0, so F_tmp = F exactly).

Cases: singular values (1, 1e-2, 1e-3), (1, 1, 1e-3), (1.2, 1e-2, 1e-2 (1 + 1e-4)), nearly
repeated (1, 1 + 1e-6, 0.5) and the well-conditioned range of the benchmark scenes
(0.3 - 1.6).  Tolerances: reconstruction 3e-6 relative to s_0; every singular value 1e-5
relative to itself; the leak into each direction 1e-4 of its singular value.  (Without the
kernel's one-sided sweep for ill-conditioned F, the eigenvectors of F^T F formed in float32
leave the smallest singular value of the 1e-3 case 4e-5 off and a 4e-3 leak.)
"""

import numpy as np
import pytest
import torch

from genesis_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _rot(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)], -1),
        np.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)], -1),
        np.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], -1),
    ], -2)


CASES = {
    "ratio_1e-3": (1.0, 1e-2, 1e-3),
    "two_equal_one_small": (1.0, 1.0, 1e-3),
    "small_pair": (1.2, 1e-2, 1e-2 * (1 + 1e-4)),
    "nearly_repeated": (1.0, 1.0 + 1e-6, 0.5),
}


def _run(F):
    from genesis_b200.engine.runtime import runtime_from_descs

    n = F.shape[0]
    density = 96
    dx = 1.0 / density
    ks = np.stack(np.meshgrid(*[np.arange(1, 16)] * 3, indexing="ij"), -1).reshape(-1, 3)[:n]
    pos = (6 * ks + 1.5) * dx
    d = W.SceneDesc(name="svd", grid_density=density, particle_size=0.01, dt=1e-4, n_substeps=1, pos=pos,
                    vel=np.zeros((n, 3)), mat_idx=np.zeros(n, dtype=np.int64),
                    materials=[("elastoplastic", dict(use_von_mises=False, yield_lower=1.0, yield_higher=1e6))],
                    gravity=(0.0, 0.0, 0.0))
    rt = runtime_from_descs([d], use_graphs=False)
    rt.set_state(pos=pos, C_=np.zeros((n, 3, 3)), F=F)
    rt.sort()
    rt.p2g()
    st = rt.get_state(("F",))
    torch.cuda.synchronize()
    return st["F"].cpu().numpy().astype(np.float64)


def test_svd_reconstruction_on_ill_conditioned_F():
    rng = np.random.default_rng(17)
    m = 64
    names, Fs, sig = [], [], []
    for name, s in CASES.items():
        S = np.tile(np.asarray(s), (m, 1))
        names += [name] * m
        sig.append(S)
    S = rng.uniform(0.3, 1.6, size=(m, 3))
    names += ["benchmark_range"] * m
    sig.append(S)
    sig = np.concatenate(sig)
    n = sig.shape[0]
    U0, V0 = _rot(rng, n), _rot(rng, n)
    F = U0 @ (sig[:, :, None] * np.swapaxes(V0, 1, 2))
    F32 = F.astype(np.float32).astype(np.float64)  # what the kernel is given
    Fn = _run(F32)
    U, s, Vt = np.linalg.svd(F32)
    E = np.swapaxes(U, 1, 2) @ (Fn - F32) @ np.swapaxes(Vt, 1, 2)
    names = np.array(names)
    for name in list(CASES) + ["benchmark_range"]:
        sel = names == name
        rec = np.abs(Fn[sel] - F32[sel]).max() / s[sel, 0].max()
        rel = np.abs(np.diagonal(E[sel], axis1=1, axis2=2)) / s[sel]
        leak = np.abs(E[sel]) / s[sel][:, None, :]
        idx = np.arange(3)
        leak[:, idx, idx] = 0
        print(f"\n[svd] {name}: max|U S V^T - F| / s0 = {rec:.2e}; per-singular-value rel. err "
              f"{rel.max(0)}; worst leak into a direction / its s = {leak.max():.2e}")
        assert rec < 3e-6, (name, rec)
        assert rel.max() < 1e-5, (name, rel.max())
        assert leak.max() < 1e-4, (name, leak.max())
