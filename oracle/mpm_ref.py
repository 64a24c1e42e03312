"""CPU oracle for the MLS-MPM substep.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import this module,
and only as the checker.  The product path (``genesis_b200``) never calls it.

This is a numpy restatement of Genesis's MPM substep, parameterised by dtype
(float32 or float64), following the reference line by line:

* solver constants          genesis/engine/solvers/mpm_solver.py:31-78
* compute_F_tmp / svd       genesis/engine/solvers/mpm_solver.py:261-275
* p2g                       genesis/engine/solvers/mpm_solver.py:290-389
* grid op (MPM core only)   genesis/engine/couplers/legacy_coupler.py:352-375, 495-496
* g2p                       genesis/engine/solvers/mpm_solver.py:391-449
* NaN check                 genesis/engine/solvers/mpm_solver.py:451-457, 505-509
* CubeBoundary              genesis/engine/boundaries/boundaries.py:12-33
* materials                 genesis/engine/materials/MPM/{base,elastic,elasto_plastic,liquid,sand,snow}.py
* EPS                       genesis/__init__.py:205-206

Parity status: UNPINNED.  The reference runs on gstaichi (pyproject.toml:13,
gstaichi==4.5.0), which is not installed here, and the reference test-suite holds no
golden vectors for MPM (its MPM tests only check qualitative invariants).  The
oracle is therefore checked against (a) those qualitative invariants, (b) an
independent C restatement (``oracle/mpm_ref.c``), and (c) exact algebraic
identities (SVD reconstruction, partition of unity, mass/momentum conservation).

SVD convention.  ``ti.svd`` (gstaichi) follows McAdams et al. 2011, "Computing the
Singular Value Decomposition of 3x3 matrices with minimal branching and elementary
floating point operations": U and V are proper rotations, singular values are
ordered by decreasing magnitude and only the last one may be negative.  The oracle
obtains the same factorisation from LAPACK's SVD by moving any reflection into the
sign of the last singular value.
"""

from __future__ import annotations

import dataclasses
import math
from dataclasses import dataclass, field

import numpy as np

KIND_ELASTIC = 0
KIND_ELASTOPLASTIC = 1
KIND_LIQUID = 2
KIND_SAND = 3
KIND_SNOW = 4
KIND_NAMES = ("elastic", "elastoplastic", "liquid", "sand", "snow")


def lame(E: float, nu: float) -> tuple[float, float]:
    """Lame parameters (mu, lam) from E and nu (materials/MPM/base.py:61-70)."""
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return mu, lam


@dataclass
class Material:
    """Plain-data restatement of one gs.materials.MPM.* object."""

    kind: int
    E: float = 1e6
    nu: float = 0.2
    rho: float = 1000.0
    mu: float = 0.0
    lam: float = 0.0
    default_Jp: float = 1.0
    neohookean: bool = False  # Elastic(model="neohooken") (elastic.py:53-58)
    use_von_mises: bool = True  # ElastoPlastic (elasto_plastic.py:53)
    von_mises_yield_stress: float = 1e4
    yield_lower: float = 2.5e-2
    yield_higher: float = 4.5e-3
    friction_angle: float = 45.0  # Sand, degrees (sand.py:41-49)
    muscle: bool = False  # Muscle: an Elastic with actuation stress (muscle.py:8-65)
    stiffness: float = 0.0  # Muscle stiffness = E (muscle.py:54)

    @property
    def alpha(self) -> float:
        # sand.py:47-49
        sin_phi = math.sin(math.radians(self.friction_angle))
        return math.sqrt(2.0 / 3.0) * 2.0 * sin_phi / (3.0 - sin_phi)


def make_material(kind: str, **kw) -> Material:
    """Construct a Material with the reference class defaults for ``kind``.

    Defaults: Elastic E=3e5 (elastic.py:40), others E=1e6; nu=0.2 and rho=1000 for all
    (base.py:36-38).  Liquid sets mu=0 unless viscous (liquid.py:47-48).  Sand uses
    default_Jp=0 (sand.py:45).  Snow is the non-von-Mises ElastoPlastic (snow.py:50-60).
    """
    kind = kind.lower()
    muscle = kind == "muscle"
    if muscle:  # muscle.py:35-55: Elastic with E=1e6 and model "neohooken" by default
        kind = "elastic"
        kw.setdefault("E", 1e6)
        kw.setdefault("model", "neohooken")
        kw.pop("n_groups", None)
    viscous = kw.pop("viscous", False)
    model = kw.pop("model", "corotation")
    E = kw.pop("E", 3e5 if kind == "elastic" else 1e6)
    nu = kw.pop("nu", 0.2)
    mu_kw = kw.pop("mu", None)
    lam_kw = kw.pop("lam", None)
    mu, lam = lame(E, nu)
    if mu_kw is not None:
        mu = mu_kw
    if lam_kw is not None:
        lam = lam_kw
    m = Material(kind=KIND_NAMES.index(kind), E=E, nu=nu, mu=mu, lam=lam, **kw)
    if kind == "elastic":
        m.neohookean = model == "neohooken"
        if muscle:
            m.muscle = True
            m.stiffness = E
    elif kind == "liquid":
        if not viscous:
            m.mu = 0.0
    elif kind == "sand":
        m.default_Jp = 0.0
    elif kind == "snow":
        m.use_von_mises = False
    return m


@dataclass
class Params:
    """Solver constants (mpm_solver.py:31-78, simulator.py:110)."""

    grid_density: float = 64.0
    lower_bound: tuple = (0.0, 0.0, 0.0)
    upper_bound: tuple = (1.0, 1.0, 1.0)
    particle_size: float | None = None
    dt: float = 1e-4  # substep dt
    gravity: tuple = (0.0, 0.0, -9.8)
    dtype: type = np.float64
    # derived
    dx: float = field(init=False)
    inv_dx: float = field(init=False)
    lower_cell: np.ndarray = field(init=False)
    upper_cell: np.ndarray = field(init=False)
    grid_res: np.ndarray = field(init=False)
    p_vol: float = field(init=False)
    bnd_lo: np.ndarray = field(init=False)
    bnd_hi: np.ndarray = field(init=False)
    eps: float = field(init=False)

    def __post_init__(self):
        if self.particle_size is None:
            # options/solvers.py:490-491
            self.particle_size = 0.01 * 64.0 / self.grid_density
        self.dx = float(1.0 / self.grid_density)
        self.inv_dx = float(self.grid_density)
        lo = np.asarray(self.lower_bound, dtype=np.float64)
        hi = np.asarray(self.upper_bound, dtype=np.float64)
        self.lower_cell = np.round(self.grid_density * lo).astype(np.int64)
        self.upper_cell = np.round(self.grid_density * hi).astype(np.int64)
        self.grid_res = self.upper_cell - self.lower_cell + 1
        # particle volume with the 1e3 scale (mpm_solver.py:43-48)
        self.p_vol = float(self.particle_size**3) * 1e3
        pad = 3 * self.dx
        self.bnd_lo = lo + pad
        self.bnd_hi = hi - pad
        # EPS = max(1e-15, finfo.eps) (__init__.py:205-206)
        self.eps = max(1e-15, float(np.finfo(self.dtype).eps))


def particle_mass(p: Params, mat: Material) -> float:
    # _kernel_add_particles: mass = particle_volume * rho (mpm_solver.py:785), in the solver dtype
    dt = p.dtype
    return float(dt(dt(p.p_vol) * dt(mat.rho)))


def svd3(F: np.ndarray):
    """Batched SVD with the rotation convention of ti.svd (see module docstring)."""
    U, s, Vh = np.linalg.svd(F)
    V = np.swapaxes(Vh, -1, -2).copy()
    U = U.copy()
    s = s.copy()
    fu = np.linalg.det(U) < 0
    U[fu, :, 2] *= -1
    s[fu, 2] *= -1
    fv = np.linalg.det(V) < 0
    V[fv, :, 2] *= -1
    s[fv, 2] *= -1
    return U, s, V


def _diag(s):
    n = s.shape[0]
    D = np.zeros((n, 3, 3), dtype=s.dtype)
    D[:, 0, 0] = s[:, 0]
    D[:, 1, 1] = s[:, 1]
    D[:, 2, 2] = s[:, 2]
    return D


def _mT(A):
    return np.swapaxes(A, -1, -2)


def update_F_S_Jp(mat: Material, eps: float, J, F_tmp, U, S, V, Jp):
    """Return mapping per material; S is the vector of singular values."""
    dt = F_tmp.dtype.type
    k = mat.kind
    if k == KIND_ELASTIC:
        # elastic.py:62-67
        return F_tmp.copy(), S.copy(), Jp.copy()
    if k == KIND_LIQUID:
        # liquid.py:50-55
        with np.errstate(invalid="ignore"):
            c = np.power(J, dt(1.0 / 3.0))
        F_new = np.zeros_like(F_tmp)
        for d in range(3):
            F_new[:, d, d] = c
        return F_new, S.copy(), Jp.copy()
    if k == KIND_ELASTOPLASTIC and mat.use_von_mises:
        # elasto_plastic.py:70-84
        Sc = np.maximum(S, dt(0.05))
        e = np.log(Sc)
        eh = e - (e.sum(axis=1, keepdims=True) / dt(3))
        ehn = np.sqrt((eh * eh).sum(axis=1) + dt(eps))
        dg = ehn - dt(mat.von_mises_yield_stress / (2 * mat.mu))
        yields = dg > 0
        e2 = e - (dg / ehn)[:, None] * eh
        S_y = np.exp(e2)
        S_new = np.where(yields[:, None], S_y, Sc)
        F_y = U @ _diag(S_y) @ _mT(V)
        F_new = np.where(yields[:, None, None], F_y, F_tmp)
        return F_new, S_new, Jp.copy()
    if k in (KIND_ELASTOPLASTIC, KIND_SNOW):
        # elasto_plastic.py:86-90 / snow.py:62-70
        S_new = np.minimum(np.maximum(S, dt(1 - mat.yield_lower)), dt(1 + mat.yield_higher))
        F_new = U @ _diag(S_new) @ _mT(V)
        Jp_new = Jp.copy()
        if k == KIND_SNOW:
            for d in range(3):
                Jp_new = Jp_new * (S[:, d] / S_new[:, d])
        return F_new, S_new, Jp_new
    if k == KIND_SAND:
        # sand.py:51-77
        e = np.log(np.maximum(np.abs(S), dt(1e-4)))
        tr = e.sum(axis=1) + Jp
        eh = e - (tr / dt(3))[:, None]
        ehn = np.sqrt((eh * eh).sum(axis=1) + dt(eps))
        expand = tr >= 0
        c1 = dt((3 * mat.lam + 2 * mat.mu) / (2 * mat.mu))
        dg = ehn + c1 * tr * dt(mat.alpha)
        S_c = np.exp(e - (np.maximum(dt(0), dg) / ehn)[:, None] * eh)
        S_new = np.where(expand[:, None], dt(1), S_c)
        Jp_new = np.where(expand, tr, dt(0))
        F_new = U @ _diag(S_new) @ _mT(V)
        return F_new, S_new, Jp_new
    raise ValueError(f"unknown material kind {k}")


def update_stress(mat: Material, U, S_new, V, F_tmp, F_new, J, Jp_old, actu=None, mdir=None):
    s = _update_stress(mat, U, S_new, V, F_tmp, F_new, J, Jp_old)
    if mat.muscle and actu is not None:
        # muscle.py:57-65: + stiffness * actu * F_tmp (d d^T) F_tmp^T
        dt = F_tmp.dtype.type
        fd = np.einsum("nij,nj->ni", F_tmp, mdir.astype(F_tmp.dtype))
        s = s + (dt(mat.stiffness) * actu.astype(F_tmp.dtype))[:, None, None] * fd[:, :, None] * fd[:, None, :]
    return s


def _update_stress(mat: Material, U, S_new, V, F_tmp, F_new, J, Jp_old):
    dt = F_tmp.dtype.type
    n = F_tmp.shape[0]
    eye = np.broadcast_to(np.eye(3, dtype=F_tmp.dtype), (n, 3, 3))
    k = mat.kind
    mu, lam = dt(mat.mu), dt(mat.lam)
    if k == KIND_ELASTIC and mat.neohookean:
        # elastic.py:77-83
        with np.errstate(invalid="ignore", divide="ignore"):
            lj = np.log(J)
        return mu * (F_tmp @ _mT(F_tmp)) + eye * (lam * lj - mu)[:, None, None]
    if k == KIND_LIQUID:
        # liquid.py:57-64 (uses F_tmp)
        R = U @ _mT(V)
        return dt(2) * mu * (F_tmp - R) @ _mT(F_tmp) + eye * (lam * J * (J - dt(1)))[:, None, None]
    if k == KIND_SAND:
        # sand.py:79-89 (S is S_new, mpm_solver.py:335)
        with np.errstate(invalid="ignore", divide="ignore"):
            lS = np.log(S_new)
        lsum = lS.sum(axis=1)
        center = dt(2.0) * mu * lS * (dt(1) / S_new) + lam * lsum[:, None] * (dt(1) / S_new)
        return U @ _diag(center) @ _mT(V) @ _mT(F_new)
    if k == KIND_SNOW:
        # snow.py:72-81 (hardening uses the previous Jp, mpm_solver.py:329,340)
        h = np.exp(dt(10) * (dt(1.0) - Jp_old))
        muh, lamh = mu * h, lam * h
        R = U @ _mT(V)
        return (dt(2) * muh)[:, None, None] * (F_new - R) @ _mT(F_new) + eye * (lamh * J * (J - dt(1)))[:, None, None]
    # Elastic corotated (elastic.py:69-75) and ElastoPlastic (base.py:83-90)
    R = U @ _mT(V)
    return dt(2) * mu * (F_new - R) @ _mT(F_new) + eye * (lam * J * (J - dt(1)))[:, None, None]


def _weights(fx):
    dt = fx.dtype.type
    return (
        dt(0.5) * (dt(1.5) - fx) ** 2,
        dt(0.75) - (fx - dt(1)) ** 2,
        dt(0.5) * (fx - dt(0.5)) ** 2,
    )


def boundary(p: Params, pos, vel):
    """CubeBoundary.impose_pos_vel with restitution 0 (boundaries.py:23-33)."""
    dt = pos.dtype.type
    lo = p.bnd_lo.astype(pos.dtype)
    hi = p.bnd_hi.astype(pos.dtype)
    vel = vel.copy()
    for i in range(3):
        up = (pos[:, i] >= hi[i]) & (vel[:, i] >= 0)
        dn = (~up) & (pos[:, i] <= lo[i]) & (vel[:, i] <= 0)
        vel[:, i] = np.where(up | dn, vel[:, i] * dt(-0.0), vel[:, i])
    pos = np.maximum(np.minimum(pos, hi), lo)
    return pos, vel


def p2g(p: Params, mats: list[Material], st: dict):
    """compute_F_tmp + svd + p2g (mpm_solver.py:261-389).

    Returns (grid_mass[res], grid_mom[res,3], F_new, Jp_new).
    """
    dt = p.dtype
    x, v, C, F, Jp = st["x"], st["v"], st["C"], st["F"], st["Jp"]
    mat_idx, active = st["mat"], st["active"]
    free = st.get("free")
    N = x.shape[0]
    res = tuple(int(r) for r in p.grid_res)
    F_new = F.copy()
    Jp_new = Jp.copy()
    gm = np.zeros(res, dtype=np.float64)
    gp = np.zeros(res + (3,), dtype=np.float64)
    act = np.nonzero(active)[0]
    if act.size == 0:
        return gm.astype(dt), gp.astype(dt), F_new, Jp_new
    eye = np.eye(3, dtype=dt)
    sdt = dt(p.dt)
    # compute_F_tmp (mpm_solver.py:261-267)
    F_tmp = (eye + sdt * C[act]) @ F[act]
    # svd (mpm_solver.py:269-275)
    U, S, V = svd3(F_tmp)
    U, S, V = U.astype(dt), S.astype(dt), V.astype(dt)
    # J = S.determinant() with S diagonal (mpm_solver.py:305)
    J = S[:, 0] * (S[:, 1] * S[:, 2])
    stress = np.zeros((act.size, 3, 3), dtype=dt)
    Fn = np.empty_like(F_tmp)
    Jn = np.empty(act.size, dtype=dt)
    mass = np.empty(act.size, dtype=dt)
    ma = mat_idx[act]
    for mi, mat in enumerate(mats):
        sel = np.nonzero(ma == mi)[0]
        if sel.size == 0:
            continue
        f_n, s_n, j_n = update_F_S_Jp(mat, p.eps, J[sel], F_tmp[sel], U[sel], S[sel], V[sel], Jp[act][sel])
        Fn[sel] = f_n
        Jn[sel] = j_n
        actu = st["actu"][act][sel] if st.get("actu") is not None else None
        mdir = st["mdir"][act][sel] if st.get("mdir") is not None else None
        stress[sel] = update_stress(mat, U[sel], s_n, V[sel], F_tmp[sel], f_n, J[sel], Jp[act][sel], actu, mdir)
        mass[sel] = particle_mass(p, mat)
    F_new[act] = Fn
    Jp_new[act] = Jn
    # mpm_solver.py:344-345
    scale = dt(-p.dt * p.p_vol * 4 * p.inv_dx * p.inv_dx)
    affine = scale * stress + mass[:, None, None] * C[act]
    xa = x[act]
    xi = xa * dt(p.inv_dx)
    base = np.floor(xi - dt(0.5)).astype(np.int64)
    fx = xi - base.astype(dt)
    w = _weights(fx)
    mv = mass[:, None] * v[act]
    node0 = base - p.lower_cell[None, :]
    flat_size = int(np.prod(res))
    gm_f = gm.reshape(-1)
    gp_f = gp.reshape(-1, 3)
    zero_nodes = []
    nonfree = None
    if free is not None:
        nonfree = ~free[act]
    for i in range(3):
        for j in range(3):
            for k in range(3):
                off = np.array([i, j, k], dtype=dt)
                dpos = (off[None, :] - fx) * dt(p.dx)
                weight = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
                contrib = weight[:, None] * (mv + np.einsum("nij,nj->ni", affine, dpos))
                node = node0 + np.array([i, j, k])
                if np.any(node < 0) or np.any(node >= np.asarray(res)):
                    raise IndexError("particle stencil outside the grid")
                lin = np.ravel_multi_index(node.T, res)
                gm_f += np.bincount(lin, weights=(weight * mass).astype(np.float64), minlength=flat_size)
                for d in range(3):
                    gp_f[:, d] += np.bincount(lin, weights=contrib[:, d].astype(np.float64), minlength=flat_size)
                if nonfree is not None and nonfree.any():
                    zero_nodes.append(lin[nonfree])
    for zn in zero_nodes:
        gp_f[zn] = 0.0  # non-free particles zero vel_in (mpm_solver.py:388-389)
    return gm.astype(dt), gp.astype(dt), F_new, Jp_new


@dataclass
class Collider:
    """A kinematic rigid geom coupled in the grid op (legacy_coupler.py:131-343): kind
    'sphere' (data[0] = radius), 'plane' (data = unit normal, geom frame) or 'box' (data =
    half extents); pose (pos, rot world-from-geom), velocity (lin_vel of pos, ang_vel) and
    the Rigid material's coupling parameters (materials/rigid.py:46-49).  Kind 'tool' is a
    Tool entity (tool_entity/mesh.py:80-176) with its voxel grid (collide_tool)."""

    kind: str
    pos: np.ndarray
    rot: np.ndarray
    data: np.ndarray
    lin_vel: np.ndarray = field(default_factory=lambda: np.zeros(3))
    ang_vel: np.ndarray = field(default_factory=lambda: np.zeros(3))
    friction: float = 0.1
    softness: float = 0.002
    restitution: float = 0.0
    sdf: np.ndarray | None = None  # kind 'tool' / 'sdf': [rx, ry, rz] voxel signed distances
    sdf_scale: tuple = (1.0, 1.0, 1.0)  # kind 'tool' / 'sdf': voxel = sdf_scale * geom-frame point + (res - 1) / 2
    floor: float = 0.0  # kind 'tool': the tool solver's floor height
    sdf_grad: np.ndarray | None = None  # kind 'sdf': [rx, ry, rz, 3] sampled gradient
    sdf_cell: float = 1.0  # kind 'sdf': cell size
    sdf_max: float = 0.0  # kind 'sdf': largest sampled distance


def sdf_sampled(c: Collider, l, eps):
    """A geom's sampled signed distance and gradient at geom-frame points l (sdf_func_sdf /
    sdf_func_grad, utils/sdf_decomp.py:102-276): trilinear in the grid centred at c.data (the
    centre of the geom's vertex bounds, T_mesh_to_sdf of rigid_geom.py:180-185); outside it
    the proxy |voxel - centre| / cell + sdf_max and the unit direction to the centre."""
    dt = l.dtype.type
    r = np.asarray(np.shape(c.sdf))
    half = (r - 1) * dt(0.5)
    ps = (l - np.asarray(c.data, dtype=dt)) * np.asarray(c.sdf_scale, dtype=dt) + half
    dc = ps - half
    out = ((ps >= r - 1) | (ps <= 0)).any(1)
    d2 = (dc * dc).sum(1)
    sd_out = np.sqrt(d2) / dt(c.sdf_cell) + dt(c.sdf_max)
    g_out = dc / np.sqrt(d2 + dt(eps))[:, None]
    b = np.minimum(np.floor(ps).astype(np.int64), r - 2)
    b = np.clip(b, 0, r - 2)
    val = np.asarray(c.sdf, dtype=dt)
    grd = np.asarray(c.sdf_grad, dtype=dt)
    sd_in = np.zeros(len(l), dtype=dt)
    g_in = np.zeros_like(l)
    for o in range(8):
        cell = b + np.array([o >> 2, (o >> 1) & 1, o & 1])
        w = np.prod(1 - np.abs(ps - cell), axis=1)
        sd_in += w * val[cell[:, 0], cell[:, 1], cell[:, 2]]
        g_in += w[:, None] * grd[cell[:, 0], cell[:, 1], cell[:, 2]]
    return np.where(out, sd_out, sd_in), np.where(out[:, None], g_out, g_in)


def _where_pos(x):
    """max(x, 0) deciding on the real part (complex-step safe)."""
    return np.where(np.real(x) > 0, x, 0)


def tool_sdf_at(vox, pv):
    """mesh.py:89-104 (Mesh.sdf_): trilinear sample of the voxel grid vox [r, r, r] at voxel
    coordinates pv [G, 3]; 1 where floor(pv) leaves [0, r - 2].  Complex pv (the complex
    step of the adjoint oracle) is sampled with the cell and |.| decided on the real part."""
    r = vox.shape[0]
    base = np.floor(np.real(pv)).astype(np.int64)
    out = ((base >= r - 1) | (base < 0)).any(1)
    b = np.clip(base, 0, r - 2)
    sd = np.zeros(len(pv), dtype=np.result_type(pv.dtype, vox.dtype))
    for o in range(8):
        cell = b + np.array([o >> 2, (o >> 1) & 1, o & 1])
        d = pv - cell
        w = np.prod(1 - np.where(np.real(d) >= 0, d, -d), axis=1)
        sd = sd + w * vox[cell[:, 0], cell[:, 1], cell[:, 2]]
    return np.where(out, 1.0, sd)


def collide_tool(c: Collider, eps, sdt, pos, vel, tool_pos=None, tool_lin_vel=None):
    """Tool.collide (tool_entity/mesh.py:147-176) for grid nodes at pos [G, 3] with velocity
    vel [G, 3]: influence min(exp(-sd / max(EPS, softness)), 1), acting where sd <= 0 or the
    influence is above 0.1; the body point's velocity from the pose one substep later
    (vel_collider, mesh.py:139-145, the origin kept above the tool solver's floor); the
    normal from central differences of 1e-2 voxel, normalised in the voxel frame, mapped to
    the world and normalised again (mesh.py:107-137); friction on the tangential part.
    tool_pos / tool_lin_vel replace c.pos / c.lin_vel (the adjoint oracle passes complex
    values for its complex-step derivatives; every branch is decided on real parts)."""
    tp = np.asarray(c.pos if tool_pos is None else tool_pos)
    tl = np.asarray(c.lin_vel if tool_lin_vel is None else tool_lin_vel)
    Rm = np.asarray(c.rot, dtype=np.float64)
    sc = np.asarray(c.sdf_scale, dtype=np.float64)
    vox = np.asarray(c.sdf, dtype=np.float64)
    half = 0.5 * (vox.shape[0] - 1)
    q = pos - tp[None, :]
    pv = (q @ Rm) * sc[None, :] + half
    sd = tool_sdf_at(vox, pv)
    e = np.exp(-sd / max(eps, c.softness))
    infl = np.where(np.real(e) < 1, e, 1.0)
    near = (np.real(sd) <= 0) | (np.real(infl) > 0.1)
    w = np.asarray(c.ang_vel, dtype=np.float64) * sdt
    th = float(np.linalg.norm(w))
    d = np.zeros_like(q)
    if th > 0:
        k = np.broadcast_to(w / th, q.shape)
        kq = np.cross(k, q)
        d = np.sin(th) * kq + 2 * np.sin(th / 2) ** 2 * np.cross(k, kq)
    dpos = tl * sdt
    if np.real(tp[2] + dpos[2]) < c.floor:
        dpos = np.array([dpos[0], dpos[1], c.floor - tp[2]])
    vc = (d + dpos[None, :]) / sdt
    rv = vel - vc
    cols = []
    for i in range(3):
        a, b = pv.copy(), pv.copy()
        a[:, i] += 1e-2
        b[:, i] -= 1e-2
        cols.append((tool_sdf_at(vox, a) - tool_sdf_at(vox, b)) / 2e-2)
    nv = np.stack(cols, 1)
    nv = nv / np.sqrt((nv * nv).sum(1) + eps)[:, None]
    n = (nv / sc[None, :]) @ Rm.T
    n = n / np.sqrt((n * n).sum(1) + eps)[:, None]
    rn = (rv * n).sum(1)
    rt = rv - rn[:, None] * n
    rtn = np.sqrt((rt * rt).sum(1) + eps)
    s_ = _where_pos(rtn + rn * c.friction) / rtn
    nvel = vc + rt * (s_ * infl)[:, None] + rv * (1 - infl)[:, None]
    hit = near & (np.real(rn) < 0)
    return np.where(hit[:, None], nvel, vel)


def collide_rigid(c: Collider, eps, sdt, pos, vel, mass):
    """_func_collide_with_rigid_geom + _func_collide_in_rigid_geom for grid nodes at pos
    (legacy_coupler.py:166-343); sphere and plane SDFs as utils/sdf_decomp.py:91-98, kind
    'sdf' through its sampled grid (sdf_sampled), kind 'box' the exact box distance.  Returns
    (new velocity, force, torque about c.pos).  A complex vel (the adjoint oracle's complex
    step) leaves the geometry real."""
    dt = np.float64 if np.iscomplexobj(vel) else vel.dtype.type
    q = pos - np.asarray(c.pos, dtype=dt)
    R = np.asarray(c.rot, dtype=dt)
    data = np.asarray(c.data, dtype=dt)
    if c.kind == "sphere":
        sd = np.linalg.norm(q, axis=1) - data[0]
        g = q / np.sqrt((q * q).sum(1) + dt(eps))[:, None]
    else:
        l = q @ R  # geom frame: R^T q per row
        if c.kind == "plane":
            sd = l @ data
            gl = np.broadcast_to(data, l.shape)
        elif c.kind == "sdf":
            sd, gl = sdf_sampled(c, l, eps)
        else:
            d = np.abs(l) - data
            o = np.maximum(d, 0)
            out = np.sqrt((o * o).sum(1))
            sd = out + np.minimum(d.max(1), 0)
            with np.errstate(invalid="ignore", divide="ignore"):
                g_out = np.copysign(o, l) / out[:, None]
            a = d.argmax(1)
            g_in = np.zeros_like(l)
            g_in[np.arange(len(l)), a] = np.copysign(dt(1), l[np.arange(len(l)), a])
            gl = np.where((out > 0)[:, None], g_out, g_in)
        g = gl @ R.T
    with np.errstate(over="ignore"):
        infl = np.minimum(np.exp(-sd / max(1e-10, c.softness)), dt(1)).astype(dt)
    n = g / np.sqrt((g * g).sum(1) + dt(eps))[:, None]
    vr = np.asarray(c.lin_vel, dtype=dt)[None, :] + np.cross(np.asarray(c.ang_vel, dtype=dt)[None, :], q)
    dt = vel.dtype.type  # the response in vel's type
    rv = vel - vr
    rn = (rv * n).sum(1)
    hit = (infl > 0.1) & (np.real(rn) < 0)
    rt = rv - rn[:, None] * n
    rtn = np.sqrt((rt * rt).sum(1) + dt(eps))
    sc = _where_pos(rtn + rn * dt(c.friction)) / rtn
    rnew = rt * sc[:, None] - n * (rn * dt(c.restitution))[:, None]
    nv = vr + rnew * infl[:, None] + rv * (dt(1) - infl)[:, None]
    out_v = np.where(hit[:, None], nv, vel)
    f = -(mass[:, None] * (out_v - vel)) / dt(sdt)
    return out_v, f.sum(0), np.cross(q, f).sum(0)


def advance_colliders(p: Params, colliders):
    """Constant-velocity kinematic motion over one substep (pos += v dt, rot = exp(w dt) rot)."""
    out = []
    for c in colliders:
        w = np.asarray(c.ang_vel, dtype=np.float64) * p.dt
        th = np.linalg.norm(w)
        R = np.asarray(c.rot, dtype=np.float64)
        if th > 0:
            k = w / th
            K = np.array([[0, -k[2], k[1]], [k[2], 0, -k[0]], [-k[1], k[0], 0]])
            R = (np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K) @ R
        pos = np.asarray(c.pos) + np.asarray(c.lin_vel) * p.dt
        if c.kind == "tool":  # the tool solver's FloorBoundary.impose_pos (tool_entity.py:180-182)
            pos[2] = max(pos[2], c.floor)
        out.append(dataclasses.replace(c, pos=pos, rot=R))
    return out


# ---------------------------------------------------------------- external force fields
# engine/force_fields.py: what each class's __init__ derives from its arguments, and _get_acc.


def _perlin_perm(seed, seed_offset, wrap_size=256):
    """PerlinNoiseField's table (force_fields.py:447-460)."""
    perm = np.arange(wrap_size, dtype=np.int64)
    if seed is not None:
        np.random.RandomState(seed + seed_offset).shuffle(perm)
    return np.concatenate([perm, perm])


def make_force_field(name: str, **kw) -> dict:
    """An active field with the reference constructor's arguments (force_fields.py:49-421)."""
    f = dict(name=name)
    if name in ("Constant", "Wind"):
        d = np.asarray(kw.get("direction", (1, 0, 0)), dtype=np.float64)
        f.update(direction=d / np.linalg.norm(d), strength=kw.get("strength", 1.0))
        if name == "Wind":
            f.update(radius=kw.get("radius", 1), center=np.asarray(kw.get("center", (0, 0, 0)), dtype=np.float64))
    elif name == "Point":
        f.update(strength=kw.get("strength", 1.0), position=np.asarray(kw.get("position", (0, 0, 0)), float),
                 falloff_pow=kw.get("falloff_pow", 0.0), flow=kw.get("flow", 1.0))
    elif name == "Drag":
        f.update(linear=kw.get("linear", 0.0), quadratic=kw.get("quadratic", 0.0))
    elif name == "Vortex":
        f.update(center=np.asarray(kw.get("center", (0.0, 0.0, 0.0)), float),
                 sp=kw.get("strength_perpendicular", 20.0), sr=kw.get("strength_radial", 0.0),
                 falloff_pow=kw.get("falloff_pow", 2.0), falloff_min=kw.get("falloff_min", 0.01),
                 falloff_max=kw.get("falloff_max", np.inf), damping=kw.get("damping", 0.0))
    elif name == "Turbulence":
        seed = kw.get("seed")
        f.update(strength=kw.get("strength", 1.0), frequency=kw.get("frequency", 3), flow=kw.get("flow", 0.0),
                 perms=[_perlin_perm(seed, k) for k in range(3)])
    else:
        raise ValueError(f"no oracle for force field {name}")
    return f


def _perlin(P, freq, x, y, z):
    """PerlinNoiseField._noise (force_fields.py:495-540) at arrays of points."""
    x, y, z = x * freq, y * freq, z * freq
    fx, fy, fz = np.floor(x), np.floor(y), np.floor(z)
    X, Y, Z = fx.astype(np.int64) & 255, fy.astype(np.int64) & 255, fz.astype(np.int64) & 255
    x, y, z = x - fx, y - fy, z - fz
    fade = lambda t: t * t * t * (t * (t * 6 - 15) + 10)
    lerp = lambda t, a, b: a + t * (b - a)

    def grad(h, x, y, z):
        h = h & 15
        u = np.where(h < 8, x, y)
        v = np.where(h < 4, y, np.where((h == 12) | (h == 14), x, z))
        return np.where(h & 1, -u, u) + np.where(h & 2, -v, v)

    u, v, w = fade(x), fade(y), fade(z)
    A = P[X] + Y
    AA, AB = P[A] + Z, P[A + 1] + Z
    B = P[X + 1] + Y
    BA, BB = P[B] + Z, P[B + 1] + Z
    return lerp(w, lerp(v, lerp(u, grad(P[AA], x, y, z), grad(P[BA], x - 1, y, z)),
                        lerp(u, grad(P[AB], x, y - 1, z), grad(P[BB], x - 1, y - 1, z))),
                lerp(v, lerp(u, grad(P[AA + 1], x, y, z - 1), grad(P[BA + 1], x - 1, y, z - 1)),
                        lerp(u, grad(P[AB + 1], x, y - 1, z - 1), grad(P[BB + 1], x - 1, y - 1, z - 1))))


def force_field_acc(f: dict, pos, vel, eps):
    """_get_acc of an active field at points pos [G, 3] with velocities vel [G, 3]."""
    n = f["name"]
    if n == "Constant":
        return np.broadcast_to(f["direction"] * f["strength"], pos.shape).copy()
    if n == "Wind":
        dist = np.linalg.norm(np.cross(pos - f["center"], f["direction"]), axis=1)
        return np.where((dist > f["radius"])[:, None], 0.0, f["direction"] * f["strength"])
    if n == "Point":
        r = pos - f["position"]
        rad = np.sqrt((r * r).sum(1) + eps)
        acc = f["strength"] * r / rad[:, None]
        acc = acc + (acc - vel) * f["flow"]
        return acc * (1.0 / (rad + 1.0) ** f["falloff_pow"])[:, None]
    if n == "Drag":  # |v| as sqrt(v.v), analytic for the adjoint oracle's complex steps
        return -f["linear"] * vel - f["quadratic"] * np.sqrt((vel * vel).sum(1))[:, None] * vel
    if n == "Vortex":
        rx, ry = pos[:, 0] - f["center"][0], pos[:, 1] - f["center"][1]
        rho = np.sqrt(rx * rx + ry * ry)
        with np.errstate(divide="ignore", invalid="ignore"):
            fo = np.where(rho < f["falloff_min"], 1.0,
                          np.where(rho < f["falloff_max"], 1.0 / (rho - f["falloff_min"] + 1.0) ** f["falloff_pow"], 0.0))
        perp = np.stack([-ry, rx, np.zeros_like(rx)], 1)
        radial = -np.stack([rx, ry, np.zeros_like(rx)], 1)
        return fo[:, None] * (f["sp"] * perp + f["sr"] * radial) - f["damping"] * vel
    if n == "Turbulence":
        acc = np.stack([_perlin(P, f["frequency"], pos[:, 0], pos[:, 1], pos[:, 2]) for P in f["perms"]], 1)
        acc = acc * f["strength"]
        return acc + (acc - vel) * f["flow"]
    raise ValueError(n)


def grid_op(p: Params, gm, gp, colliders=None, forces=None, force_fields=None):
    """MPM core of LegacyCoupler.mpm_grid_op (legacy_coupler.py:364-375, 495-496), with the
    rigid coupling of :385-397 for kinematic colliders (forces, if a list, receives one
    (force, torque) pair per collider)."""
    dt = p.dtype
    res = gm.shape
    vel = np.zeros(res + (3,), dtype=dt)
    act = gm > dt(p.eps)
    m = gm[act]
    v = (dt(1) / m)[:, None] * gp[act]
    v = v + dt(p.dt) * np.asarray(p.gravity, dtype=dt)[None, :]
    idx = np.argwhere(act)
    pos = (idx + p.lower_cell[None, :]).astype(dt) * dt(p.dx)
    for f in force_fields or []:  # external force fields (legacy_coupler.py:377-379)
        v = (v + force_field_acc(f, pos.astype(np.float64), v.astype(np.float64), p.eps) * p.dt).astype(dt)
    for c in colliders or []:  # MPM <-> Tool first (legacy_coupler.py:381-383)
        if c.kind == "tool":
            v = collide_tool(c, p.eps, p.dt, pos, v).astype(dt)
    for c in colliders or []:
        if c.kind == "tool":
            if forces is not None:
                forces.append((np.zeros(3), np.zeros(3)))
            continue
        v, f, t = collide_rigid(c, p.eps, p.dt, pos, v, (m / dt(1e3)).astype(dt))
        if forces is not None:
            forces.append((f, t))
    _, v = boundary(p, pos, v)
    vel[act] = v
    return vel


def g2p(p: Params, st: dict, vel):
    """g2p (mpm_solver.py:391-449); returns new x, v, C for active particles."""
    dt = p.dtype
    x, v, C = st["x"], st["v"], st["C"]
    active = st["active"]
    res = vel.shape[:3]
    xn, vn, Cn = x.copy(), v.copy(), C.copy()
    act = np.nonzero(active)[0]
    if act.size == 0:
        return xn, vn, Cn
    xa = x[act]
    xi = xa * dt(p.inv_dx)
    base = np.floor(xi - dt(0.5)).astype(np.int64)
    fx = xi - base.astype(dt)
    w = _weights(fx)
    node0 = base - p.lower_cell[None, :]
    new_v = np.zeros((act.size, 3), dtype=dt)
    new_C = np.zeros((act.size, 3, 3), dtype=dt)
    vflat = vel.reshape(-1, 3)
    c4 = dt(4 * p.inv_dx)
    for i in range(3):
        for j in range(3):
            for k in range(3):
                off = np.array([i, j, k], dtype=dt)
                dpos = off[None, :] - fx
                weight = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
                node = node0 + np.array([i, j, k])
                lin = np.ravel_multi_index(node.T, res)
                gv = vflat[lin]
                new_v += weight[:, None] * gv
                new_C += (c4 * weight)[:, None, None] * (gv[:, :, None] * dpos[:, None, :])
    new_x = xa + dt(p.dt) * new_v
    new_x, new_v = boundary(p, new_x, new_v)
    xn[act] = new_x
    vn[act] = new_v
    Cn[act] = new_C
    return xn, vn, Cn


def substep(p: Params, mats: list[Material], st: dict, return_grid: bool = False):
    """One full substep: p2g, grid op, g2p.  ``st`` is not modified."""
    gm, gp, F_new, Jp_new = p2g(p, mats, st)
    colliders = st.get("colliders")
    vel = grid_op(p, gm, gp, colliders, force_fields=st.get("force_fields"))
    xn, vn, Cn = g2p(p, st, vel)
    out = dict(st)
    out.update(x=xn, v=vn, C=Cn, F=F_new, Jp=Jp_new)
    if colliders:
        out["colliders"] = advance_colliders(p, colliders)
    if np.isnan(xn).any():
        raise FloatingPointError("NaN detected in MPM states (mpm_solver.py:505-509)")
    if return_grid:
        return out, (gm, gp, vel)
    return out


def make_state(x, mats: list[Material], mat_idx, dtype, v=None, active=None):
    """Fresh particle state as _kernel_add_particles / set_particles_pos leave it
    (mpm_solver.py:768-801, 803-822): v=0 unless given, F=I, C=0, Jp=default_Jp."""
    x = np.asarray(x, dtype=dtype)
    N = x.shape[0]
    mat_idx = np.asarray(mat_idx, dtype=np.int64)
    st = dict(
        x=x.copy(),
        v=np.zeros((N, 3), dtype=dtype) if v is None else np.asarray(v, dtype=dtype).copy(),
        C=np.zeros((N, 3, 3), dtype=dtype),
        F=np.broadcast_to(np.eye(3, dtype=dtype), (N, 3, 3)).copy(),
        Jp=np.array([mats[m].default_Jp for m in mat_idx], dtype=dtype) if N else np.zeros(0, dtype),
        mat=mat_idx,
        active=np.ones(N, dtype=bool) if active is None else np.asarray(active, dtype=bool).copy(),
    )
    return st


def run(p: Params, mats, st, n_substeps: int):
    for _ in range(n_substeps):
        st = substep(p, mats, st)
    return st
