"""Reverse-mode adjoint of one MPM substep (Elastic, corotated) -- TEST INFRASTRUCTURE ONLY.

numpy restatement of the hand-derived adjoint that the CUDA kernels implement, used to
check them.  It differentiates exactly the forward of ``mpm_ref.substep`` for Elastic
materials with per-particle Lame parameters:

  F_tmp = (I + dt C) F                                  mpm_solver.py:264-266
  F_tmp = U S V^T, R = U V^T, J = det F_tmp             mpm_solver.py:273, 305
  P = 2 mu (F_tmp - R) F_tmp^T + lam J (J - 1) I        elastic.py:70-75
  A = s P + m C,  s = -dt vol 4 inv_dx^2                mpm_solver.py:344-345
  grid: m_i = sum w m,  p_i = sum w (m v + A d_i)       mpm_solver.py:347-386
  v_i = bc(p_i / m_i + dt g)                            legacy_coupler.py:369-372, 495-496
  v' = sum w v_i,  C' = c sum w v_i u_i^T,  x' = x + dt v', then the boundary
                                                        mpm_solver.py:396-437
with d_i = (off - fx) dx = x_i - x_p, u_i = off - fx (cell units), c = 4 inv_dx.

The polar-rotation part of the SVD backward uses the closed form
  Fbar += U [(M_ij - M_ji) / (s_i + s_j)] V^T,   M = U^T Rbar V,
which is what the reference's backward_svd (mpm_solver.py:1112-1129, the PyTorch SVD
adjoint) reduces to for R = U V^T, written without the 1 / (s_j^2 - s_i^2) factors that
its signmax(., 1e-6) guard clamps when singular values nearly coincide.
"""

from __future__ import annotations

import numpy as np

from . import mpm_ref as R


def _mT(A):
    return np.swapaxes(A, -1, -2)


def backward_svd(gU, gS, gV, U, S, V):
    """Restatement of the reference's backward_svd (mpm_solver.py:1106-1129, the PyTorch
    SVD adjoint), batched over the leading axis: given the adjoints of U, S (a 3x3 matrix,
    diagonal in the forward) and V of F = U S V^T, the adjoint of F is
      U [(F o (U^T gU - gU^T U)) S] V^T + U [S ((F o (V^T gV - gV^T V)) V^T)] + U gS V^T,
    with F_ij = 1 / signmax(s_j^2 - s_i^2, 1e-6) off the diagonal and 0 on it, s_i = S_ii,
    signmax(a, e) = sign(a) max(|a|, e) (sign(0) = +1)."""
    vt, ut = _mT(V), _mT(U)
    s2 = np.diagonal(S, axis1=-2, axis2=-1) ** 2
    diff = s2[..., None, :] - s2[..., :, None]  # [i, j] = s_j^2 - s_i^2
    sm = np.where(diff >= 0, 1.0, -1.0) * np.maximum(np.abs(diff), 1e-6)
    Fm = 1.0 / sm
    idx = np.arange(3)
    Fm[..., idx, idx] = 0.0
    s_term = U @ gS @ vt
    u_term = U @ ((Fm * (ut @ gU - _mT(gU) @ U)) @ S) @ vt
    v_term = U @ (S @ ((Fm * (vt @ gV - _mT(gV) @ V)) @ vt))
    return u_term + v_term + s_term


def _weights_and_grads(fx):
    w = [0.5 * (1.5 - fx) ** 2, 0.75 - (fx - 1.0) ** 2, 0.5 * (fx - 0.5) ** 2]
    dw = [-(1.5 - fx), -2.0 * (fx - 1.0), fx - 0.5]
    return w, dw


def _stencil(p, x):
    xi = x * p.inv_dx
    base = np.floor(xi - 0.5).astype(np.int64)
    fx = xi - base
    w, dw = _weights_and_grads(fx)
    node0 = base - p.lower_cell[None, :]
    return base, fx, w, dw, node0


def _offsets():
    for i in range(3):
        for j in range(3):
            for k in range(3):
                yield i, j, k


def forward(p, st, mu, lam, mass):
    """One substep for all (active, Elastic) particles with per-particle mu/lam; returns the
    new state and the intermediates the adjoint needs."""
    x, v, C, F = st["x"], st["v"], st["C"], st["F"]
    n = x.shape[0]
    eye = np.eye(3)
    Ft = (eye + p.dt * C) @ F
    U, S, V = R.svd3(Ft)
    Rm = U @ _mT(V)
    J = np.linalg.det(Ft)
    P = 2 * mu[:, None, None] * (Ft - Rm) @ _mT(Ft) + (lam * J * (J - 1))[:, None, None] * eye
    s = -p.dt * p.p_vol * 4 * p.inv_dx * p.inv_dx
    A = s * P + mass[:, None, None] * C
    base, fx, w, dw, node0 = _stencil(p, x)
    res = tuple(int(r) for r in p.grid_res)
    G = int(np.prod(res))
    gm = np.zeros(G)
    gp = np.zeros((G, 3))
    lin_all = []
    for i, j, k in _offsets():
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        d = (off[None, :] - fx) * p.dx
        lin = np.ravel_multi_index((node0 + off).T, res)
        lin_all.append(lin)
        gm += np.bincount(lin, weights=wt * mass, minlength=G)
        contrib = wt[:, None] * (mass[:, None] * v + np.einsum("nij,nj->ni", A, d))
        for c in range(3):
            gp[:, c] += np.bincount(lin, weights=contrib[:, c], minlength=G)
    # grid op
    act = gm > p.eps
    vg = np.zeros((G, 3))
    vg[act] = gp[act] / gm[act][:, None] + p.dt * np.asarray(p.gravity)[None, :]
    idx = np.array(np.unravel_index(np.arange(G), res)).T
    gpos = (idx + p.lower_cell[None, :]) * p.dx
    gmask = np.ones((G, 3))
    for c in range(3):
        up = (gpos[:, c] >= p.bnd_hi[c]) & (vg[:, c] >= 0)
        dn = (~up) & (gpos[:, c] <= p.bnd_lo[c]) & (vg[:, c] <= 0)
        gmask[:, c] = np.where(up | dn, 0.0, 1.0)
    gmask[~act] = 0.0
    vh = vg * gmask
    # g2p
    c4 = 4 * p.inv_dx
    nv = np.zeros((n, 3))
    nC = np.zeros((n, 3, 3))
    for (i, j, k), lin in zip(_offsets(), lin_all):
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        u = off[None, :] - fx
        nv += wt[:, None] * vh[lin]
        nC += (c4 * wt)[:, None, None] * vh[lin][:, :, None] * u[:, None, :]
    xs = x + p.dt * nv
    pmask = np.ones((n, 3))
    vmask = np.ones((n, 3))
    for c in range(3):
        up = (xs[:, c] >= p.bnd_hi[c]) & (nv[:, c] >= 0)
        dn = (~up) & (xs[:, c] <= p.bnd_lo[c]) & (nv[:, c] <= 0)
        vmask[:, c] = np.where(up | dn, 0.0, 1.0)
        pmask[:, c] = np.where((xs[:, c] > p.bnd_hi[c]) | (xs[:, c] < p.bnd_lo[c]), 0.0, 1.0)
    xn = np.clip(xs, p.bnd_lo, p.bnd_hi)
    out = dict(st)
    out.update(x=xn, v=nv * vmask, C=nC, F=Ft)
    inter = dict(Ft=Ft, U=U, S=S, V=V, Rm=Rm, J=J, P=P, A=A, fx=fx, w=w, dw=dw, lin=lin_all, gm=gm, gp=gp,
                 vh=vh, gmask=gmask, act=act, nv=nv, pmask=pmask, vmask=vmask, s=s)
    return out, inter


def backward(p, st, mu, lam, mass, inter, adj):
    """adj: dict with x, v, C, F adjoints of the substep's output.  Returns the adjoints of
    its input state and of mu, lam."""
    x, v, C, F = st["x"], st["v"], st["C"], st["F"]
    n = x.shape[0]
    G = inter["gm"].shape[0]
    fx, w, dw = inter["fx"], inter["w"], inter["dw"]
    c4 = 4 * p.inv_dx
    # ---- g2p adjoint
    gx = adj["x"] * inter["pmask"]
    vbar = adj["v"] * inter["vmask"] + p.dt * gx
    Cbar = adj["C"]
    xbar = gx.copy()
    vh_bar = np.zeros((G, 3))
    for (i, j, k), lin in zip(_offsets(), inter["lin"]):
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        gw = np.stack([dw[i][:, 0] * w[j][:, 1] * w[k][:, 2], w[i][:, 0] * dw[j][:, 1] * w[k][:, 2],
                       w[i][:, 0] * w[j][:, 1] * dw[k][:, 2]], 1) * p.inv_dx
        u = off[None, :] - fx
        vh = inter["vh"][lin]
        Cu = np.einsum("nij,nj->ni", Cbar, u)
        contrib = wt[:, None] * vbar + (c4 * wt)[:, None] * Cu
        for c in range(3):
            vh_bar[:, c] += np.bincount(lin, weights=contrib[:, c], minlength=G)
        wbar = (vbar * vh).sum(1) + c4 * (vh * Cu).sum(1)
        ubar = (c4 * wt)[:, None] * np.einsum("nji,nj->ni", Cbar, vh)
        xbar += wbar[:, None] * gw - p.inv_dx * ubar
    # ---- grid op adjoint
    vg_bar = vh_bar * inter["gmask"]
    act = inter["act"]
    pbar = np.zeros((G, 3))
    mbar = np.zeros(G)
    pbar[act] = vg_bar[act] / inter["gm"][act][:, None]
    mbar[act] = -(vg_bar[act] * inter["gp"][act]).sum(1) / inter["gm"][act] ** 2
    # ---- p2g adjoint
    A = inter["A"]
    Abar = np.zeros((n, 3, 3))
    vbar_n = np.zeros((n, 3))
    for (i, j, k), lin in zip(_offsets(), inter["lin"]):
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        gw = np.stack([dw[i][:, 0] * w[j][:, 1] * w[k][:, 2], w[i][:, 0] * dw[j][:, 1] * w[k][:, 2],
                       w[i][:, 0] * w[j][:, 1] * dw[k][:, 2]], 1) * p.inv_dx
        d = (off[None, :] - fx) * p.dx
        pb = pbar[lin]
        mb = mbar[lin]
        q = mass[:, None] * v + np.einsum("nij,nj->ni", A, d)
        wbar = mb * mass + (pb * q).sum(1)
        vbar_n += (wt * mass)[:, None] * pb
        Abar += wt[:, None, None] * pb[:, :, None] * d[:, None, :]
        xbar += wbar[:, None] * gw - wt[:, None] * np.einsum("nji,nj->ni", A, pb)
    Pbar = inter["s"] * Abar
    Cbar_n = mass[:, None, None] * Abar
    Ft, U, S, V, Rm, J = inter["Ft"], inter["U"], inter["S"], inter["V"], inter["Rm"], inter["J"]
    D = Ft - Rm
    mu_bar = 2 * np.einsum("nij,nij->n", Pbar, D @ _mT(Ft))
    trP = np.trace(Pbar, axis1=1, axis2=2)
    lam_bar = trP * J * (J - 1)
    Ft_bar = 2 * mu[:, None, None] * (Pbar @ Ft + _mT(Pbar) @ D)
    Rbar = -2 * mu[:, None, None] * Pbar @ Ft
    Jbar = lam * (2 * J - 1) * trP
    Ft_bar += Jbar[:, None, None] * J[:, None, None] * np.linalg.inv(_mT(Ft))
    M = _mT(U) @ Rbar @ V
    den = S[:, :, None] + S[:, None, :]
    X = (M - _mT(M)) / np.where(np.abs(den) > 1e-12, den, 1e-12)
    Ft_bar += U @ X @ _mT(V)
    Ft_bar += adj["F"]  # F_new = F_tmp for Elastic
    eye = np.eye(3)
    F_bar_n = _mT(eye + p.dt * C) @ Ft_bar
    Cbar_n += p.dt * Ft_bar @ _mT(F)
    return dict(x=xbar, v=vbar_n, C=Cbar_n, F=F_bar_n), mu_bar, lam_bar


def lame_of_E(E, nu):
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return mu, lam


def rollout_loss_and_grad(p, st0, E, nu, mass, n_substeps, target):
    """loss = |mean(x_T) - target|^2 and its gradient w.r.t. the initial velocity (summed
    over particles, i.e. w.r.t. a uniform v0) and per-particle E, storing every state."""
    mu, lam = lame_of_E(E, nu)
    states, inters = [st0], []
    st = st0
    for _ in range(n_substeps):
        st, it = forward(p, st, mu, lam, mass)
        states.append(st)
        inters.append(it)
    n = st0["x"].shape[0]
    xm = states[-1]["x"].mean(0)
    loss = float(((xm - target) ** 2).sum())
    adj = dict(x=np.tile(2 * (xm - target) / n, (n, 1)), v=np.zeros((n, 3)), C=np.zeros((n, 3, 3)),
               F=np.zeros((n, 3, 3)))
    mu_bar = np.zeros(n)
    lam_bar = np.zeros(n)
    for t in range(n_substeps - 1, -1, -1):
        adj, mb, lb = backward(p, states[t], mu, lam, mass, inters[t], adj)
        mu_bar += mb
        lam_bar += lb
    E_bar = mu_bar / (2.0 * (1.0 + nu)) + lam_bar * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return loss, adj["v"].sum(0), E_bar, adj


def rollout_loss(p, st0, E, nu, mass, n_substeps, target):
    mu, lam = lame_of_E(E, nu)
    st = st0
    for _ in range(n_substeps):
        st, _ = forward(p, st, mu, lam, mass)
    return float(((st["x"].mean(0) - target) ** 2).sum())


# ---------------------------------------------------------------- every MPM material
# The reference differentiates p2g with gstaichi autodiff: update_F_S_Jp and update_stress are
# differentiated with U, S, V, F_tmp and Jp as independent inputs (they are separate fields,
# mpm_solver.py:80-110, written by the svd kernel), and svd_grad then maps the adjoints of
# U, S, V to F_tmp through backward_svd (mpm_solver.py:1112-1129).  The restatement below
# does the same: the materials' own formulas (material_reference_form) are differentiated by
# the complex step, which is exact to float64 round-off, and backward_svd is applied as the
# reference writes it.


def _cabs(x):
    """|x|, continued analytically so that the complex step differentiates it."""
    return np.where(x.real >= 0, x, -x)


def _cmax(x, c):
    return np.where(x.real > c, x, c + 0 * x)


def _cclamp(x, lo, hi):
    return np.where(x.real < lo, lo + 0 * x, np.where(x.real > hi, hi + 0 * x, x))


def _usvt(U, s, V):
    return U @ (s[..., :, None] * _mT(V))


def material_reference_form(mat, eps, U, S, V, Ft, Jp, mu, lam, actu=None, mdir=None):
    """update_F_S_Jp + update_stress of one material, as p2g calls them (mpm_solver.py:303-345):
    J = det S; (F_new, S_new, Jp_new) = update_F_S_Jp(J, F_tmp, U, S, V, Jp); stress =
    update_stress(U, S_new, V, F_tmp, F_new, J, Jp_old, actu, m_dir).  Arrays over particles,
    S the [n, 3] diagonal, mu / lam per particle; complex inputs allowed.  Returns (F_new,
    Jp_new, stress)."""
    n = Ft.shape[0]
    eye = np.broadcast_to(np.eye(3), (n, 3, 3))
    J = S[:, 0] * (S[:, 1] * S[:, 2])  # S.determinant() of the diagonal S
    k = mat.kind
    mu3, lam3 = mu[:, None, None], lam[:, None, None]

    def corot(Fn, muc, lamc):  # base.py:86-88 / elastic.py:70-75
        return 2 * muc[:, None, None] * (Fn - U @ _mT(V)) @ _mT(Fn) + (lamc * J * (J - 1))[:, None, None] * eye

    if k == R.KIND_ELASTIC:  # elastic.py:62-83
        Fn, Jpn = Ft, Jp
        if mat.neohookean:
            P = mu3 * (Ft @ _mT(Ft)) + (lam * np.log(J) - mu)[:, None, None] * eye
        else:
            P = corot(Fn, mu, lam)
    elif k == R.KIND_LIQUID:  # liquid.py:50-64 (mu = 0 unless viscous: the caller's mu)
        c = J ** (1.0 / 3.0)
        Fn, Jpn = c[:, None, None] * eye, Jp
        P = 2 * mu3 * (Ft - U @ _mT(V)) @ _mT(Ft) + (lam * J * (J - 1))[:, None, None] * eye
    elif k == R.KIND_ELASTOPLASTIC and mat.use_von_mises:  # elasto_plastic.py:70-84
        Sc = _cmax(S, 0.05)
        e = np.log(Sc)
        eh = e - e.sum(1, keepdims=True) / 3
        ehn = np.sqrt((eh * eh).sum(1) + eps)
        dg = ehn - mat.von_mises_yield_stress / (2 * mu)
        y = dg.real > 0
        Sy = np.exp(e - (dg / ehn)[:, None] * eh)
        Fn = np.where(y[:, None, None], _usvt(U, Sy, V), Ft)
        Jpn = Jp
        P = corot(Fn, mu, lam)
    elif k == R.KIND_ELASTOPLASTIC:  # elasto_plastic.py:86-90
        Sn = _cclamp(S, 1 - mat.yield_lower, 1 + mat.yield_higher)
        Fn, Jpn = _usvt(U, Sn, V), Jp
        P = corot(Fn, mu, lam)
    elif k == R.KIND_SNOW:  # snow.py:62-81
        Sn = _cclamp(S, 1 - mat.yield_lower, 1 + mat.yield_higher)
        Jpn = Jp * (S / Sn).prod(1)
        Fn = _usvt(U, Sn, V)
        h = np.exp(10 * (1.0 - Jp))
        P = corot(Fn, mu * h, lam * h)
    else:  # sand.py:51-89
        e = np.log(_cmax(_cabs(S), 1e-4))
        tr = e.sum(1) + Jp
        eh = e - (tr / 3)[:, None]
        ehn = np.sqrt((eh * eh).sum(1) + eps)
        expand = tr.real >= 0
        dg = ehn + (3 * lam + 2 * mu) / (2 * mu) * tr * mat.alpha
        dgp = np.where(dg.real > 0, dg, 0 * dg)
        Sc = np.exp(e - (dgp / ehn)[:, None] * eh)
        Sn = np.where(expand[:, None], 1 + 0 * Sc, Sc)
        Jpn = np.where(expand, tr, 0 * tr)
        Fn = _usvt(U, Sn, V)
        lS = np.log(Sn)
        center = 2 * mu[:, None] * lS / Sn + lam[:, None] * lS.sum(1, keepdims=True) / Sn
        P = _usvt(U, center, V) @ _mT(Fn)
    if mat.muscle and actu is not None:  # muscle.py:57-65
        fd = np.einsum("nij,nj->ni", Ft, mdir)
        P = P + (mat.stiffness * actu)[:, None, None] * fd[:, :, None] * fd[:, None, :]
    return Fn, Jpn, P


def material_vjp(mat, eps, U, S, V, Ft, Jp, mu, lam, actu, mdir, Fn_bar, Jpn_bar, P_bar):
    """Adjoints of material_reference_form's inputs (F_tmp, U, S, V, Jp, mu, lam, actu) for the
    adjoints of its outputs, by the complex step (one evaluation per input scalar)."""
    h = 1e-30
    n = Ft.shape[0]
    act = actu if actu is not None else np.zeros(n)
    md = mdir if mdir is not None else np.zeros((n, 3))
    base = dict(Ft=Ft.reshape(n, 9), U=U.reshape(n, 9), S=S, V=V.reshape(n, 9), Jp=Jp[:, None], mu=mu[:, None],
                lam=lam[:, None], actu=act[:, None])
    out = {}
    for name, arr in base.items():
        bar = np.zeros(arr.shape)
        for j in range(arr.shape[1]):
            args = {k: v.astype(complex) for k, v in base.items()}
            args[name] = args[name].copy()
            args[name][:, j] += 1j * h
            Fn, Jpn, P = material_reference_form(
                mat, eps, args["U"].reshape(n, 3, 3), args["S"], args["V"].reshape(n, 3, 3),
                args["Ft"].reshape(n, 3, 3), args["Jp"][:, 0], args["mu"][:, 0], args["lam"][:, 0],
                args["actu"][:, 0] if actu is not None else None, md if actu is not None else None)
            d = (np.einsum("nij,nij->n", Fn_bar, Fn.imag) + Jpn_bar * np.asarray(Jpn).imag +
                 np.einsum("nij,nij->n", P_bar, P.imag)) / h
            bar[:, j] = d
        out[name] = bar
    return (out["Ft"].reshape(n, 3, 3), out["U"].reshape(n, 3, 3), out["S"], out["V"].reshape(n, 3, 3),
            out["Jp"][:, 0], out["mu"][:, 0], out["lam"][:, 0], out["actu"][:, 0])


def forward_materials(p, mats, st, mu, lam, colliders=None):
    """One substep of mpm_ref.substep for any mix of MPM materials (all particles active), with
    per-particle mu / lam and the grid op's kinematic colliders (tools, rigid geoms) at this
    substep's poses; returns the new state and the intermediates of backward_materials."""
    x, v, C, F, Jp = st["x"], st["v"], st["C"], st["F"], st["Jp"]
    n = x.shape[0]
    mi = np.asarray(st["mat"])
    Ft = (np.eye(3) + p.dt * C) @ F
    U, S, V = R.svd3(Ft)
    Fn = np.zeros_like(Ft)
    Jpn = np.zeros(n)
    P = np.zeros_like(Ft)
    mass = np.zeros(n)
    for k, m in enumerate(mats):
        sel = mi == k
        if not sel.any():
            continue
        actu = st["actu"][sel] if st.get("actu") is not None else None
        mdir = st["mdir"][sel] if st.get("mdir") is not None else None
        Fn[sel], Jpn[sel], P[sel] = material_reference_form(m, p.eps, U[sel], S[sel], V[sel], Ft[sel], Jp[sel],
                                                            mu[sel], lam[sel], actu, mdir)
        mass[sel] = R.particle_mass(p, m)
    s = -p.dt * p.p_vol * 4 * p.inv_dx * p.inv_dx
    A = s * P + mass[:, None, None] * C
    out, inter = _grid_and_g2p(p, st, A, mass, colliders, st.get("force_fields"))
    out.update(F=Fn, Jp=Jpn)
    inter.update(Ft=Ft, U=U, S=S, V=V, P=P, A=A, s=s, mass=mass)
    return out, inter


def _grid_and_g2p(p, st, A, mass, colliders=None, force_fields=None):
    """p2g scatter of (m v + A d), grid op (the force fields, then the colliders' responses,
    tools first, as legacy_coupler.py:377-397 orders them) and g2p of mpm_ref.substep."""
    x, v = st["x"], st["v"]
    n = x.shape[0]
    base, fx, w, dw, node0 = _stencil(p, x)
    res = tuple(int(r) for r in p.grid_res)
    G = int(np.prod(res))
    gm = np.zeros(G)
    gp = np.zeros((G, 3))
    lin_all = []
    for i, j, k in _offsets():
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        d = (off[None, :] - fx) * p.dx
        lin = np.ravel_multi_index((node0 + off).T, res)
        lin_all.append(lin)
        gm += np.bincount(lin, weights=wt * mass, minlength=G)
        contrib = wt[:, None] * (mass[:, None] * v + np.einsum("nij,nj->ni", A, d))
        for c in range(3):
            gp[:, c] += np.bincount(lin, weights=contrib[:, c], minlength=G)
    act = gm > p.eps
    vg = np.zeros((G, 3))
    vg[act] = gp[act] / gm[act][:, None] + p.dt * np.asarray(p.gravity)[None, :]
    idx = np.array(np.unravel_index(np.arange(G), res)).T
    gpos = (idx + p.lower_cell[None, :]) * p.dx
    ff_chain = []  # (field, its input velocity on the active nodes)
    if force_fields:
        va = vg[act]
        for f in force_fields:
            ff_chain.append((f, va))
            va = va + R.force_field_acc(f, gpos[act], va, p.eps) * p.dt
        vg[act] = va
    chain = []  # (collider index, collider, its input velocity on the active nodes)
    if colliders:
        va = vg[act]
        ma = gm[act] / 1e3
        order = [k for k, c in enumerate(colliders) if c.kind == "tool"] + \
                [k for k, c in enumerate(colliders) if c.kind != "tool"]
        for k in order:
            c = colliders[k]
            chain.append((k, c, va))
            if c.kind == "tool":
                va = R.collide_tool(c, p.eps, p.dt, gpos[act], va)
            else:
                va = R.collide_rigid(c, p.eps, p.dt, gpos[act], va, ma)[0]
        vg[act] = va
    gmask = np.ones((G, 3))
    for c in range(3):
        up = (gpos[:, c] >= p.bnd_hi[c]) & (vg[:, c] >= 0)
        dn = (~up) & (gpos[:, c] <= p.bnd_lo[c]) & (vg[:, c] <= 0)
        gmask[:, c] = np.where(up | dn, 0.0, 1.0)
    gmask[~act] = 0.0
    vh = vg * gmask
    c4 = 4 * p.inv_dx
    nv = np.zeros((n, 3))
    nC = np.zeros((n, 3, 3))
    for (i, j, k), lin in zip(_offsets(), lin_all):
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        u = off[None, :] - fx
        nv += wt[:, None] * vh[lin]
        nC += (c4 * wt)[:, None, None] * vh[lin][:, :, None] * u[:, None, :]
    xs = x + p.dt * nv
    pmask = np.ones((n, 3))
    vmask = np.ones((n, 3))
    for c in range(3):
        up = (xs[:, c] >= p.bnd_hi[c]) & (nv[:, c] >= 0)
        dn = (~up) & (xs[:, c] <= p.bnd_lo[c]) & (nv[:, c] <= 0)
        vmask[:, c] = np.where(up | dn, 0.0, 1.0)
        pmask[:, c] = np.where((xs[:, c] > p.bnd_hi[c]) | (xs[:, c] < p.bnd_lo[c]), 0.0, 1.0)
    out = dict(st)
    out.update(x=np.clip(xs, p.bnd_lo, p.bnd_hi), v=nv * vmask, C=nC)
    inter = dict(fx=fx, w=w, dw=dw, lin=lin_all, gm=gm, gp=gp, vh=vh, gmask=gmask, act=act, nv=nv, pmask=pmask,
                 vmask=vmask, chain=chain, gpos=gpos, n_colliders=len(colliders or []), ff_chain=ff_chain)
    return out, inter


def force_field_vjp(p, f, pos, vin, vbar, h=1e-30):
    """Adjoint of v + acc(pos, v) dt with respect to v at nodes pos, by complex steps."""
    out = np.zeros_like(vin)
    for k in range(3):
        vv = vin.astype(np.complex128)
        vv[:, k] += 1j * h
        dv = vv + R.force_field_acc(f, pos, vv, p.eps) * p.dt
        out[:, k] = (np.imag(dv) / h * vbar).sum(1)
    return out


def collider_vjp(p, c, pos, vin, vbar, mass=None, h=1e-30):
    """Adjoint of one collider's response at grid nodes pos [G, 3] (input velocity vin [G, 3],
    output adjoint vbar [G, 3]), by complex-step derivatives (exact to round-off, every branch
    taken on real parts): returns (vin_bar [G, 3], pos_bar [3], lin_vel_bar [3]).  For a tool,
    pos_bar / lin_vel_bar are the derivatives with respect to its position and linear
    velocity at this substep (its normal, influence and vel_collider all depend on them); a
    rigid geom's pose is taken as given (zero)."""
    G = len(vin)
    vin_bar = np.zeros((G, 3))
    pos_bar = np.zeros(3)
    lin_bar = np.zeros(3)

    def resp(vv, tp=None, tl=None):
        if c.kind == "tool":
            return R.collide_tool(c, p.eps, p.dt, pos, vv, tool_pos=tp, tool_lin_vel=tl)
        return R.collide_rigid(c, p.eps, p.dt, pos, vv, mass)[0]

    for k in range(3):
        vv = vin.astype(np.complex128)
        vv[:, k] += 1j * h
        vin_bar[:, k] = (np.imag(resp(vv)) / h * vbar).sum(1)
    if c.kind == "tool":
        for k in range(3):
            tp = np.asarray(c.pos, dtype=np.complex128).copy()
            tp[k] += 1j * h
            pos_bar[k] = (np.imag(resp(vin.astype(np.complex128), tp=tp)) / h * vbar).sum()
            tl = np.asarray(c.lin_vel, dtype=np.complex128).copy()
            tl[k] += 1j * h
            lin_bar[k] = (np.imag(resp(vin.astype(np.complex128), tl=tl)) / h * vbar).sum()
    return vin_bar, pos_bar, lin_bar


def backward_materials(p, mats, st, mu, lam, inter, adj):
    """adj: adjoints (x, v, C, F, Jp) of the substep's output.  Returns the adjoints of its
    input state (x, v, C, F, Jp) and of mu, lam and (Muscle) actu, per particle."""
    x, v, C, F = st["x"], st["v"], st["C"], st["F"]
    n = x.shape[0]
    G = inter["gm"].shape[0]
    fx, w, dw = inter["fx"], inter["w"], inter["dw"]
    c4 = 4 * p.inv_dx
    mass = inter["mass"]
    # g2p
    gx = adj["x"] * inter["pmask"]
    vbar = adj["v"] * inter["vmask"] + p.dt * gx
    Cbar = adj["C"]
    xbar = gx.copy()
    vh_bar = np.zeros((G, 3))
    for (i, j, k), lin in zip(_offsets(), inter["lin"]):
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        gw = np.stack([dw[i][:, 0] * w[j][:, 1] * w[k][:, 2], w[i][:, 0] * dw[j][:, 1] * w[k][:, 2],
                       w[i][:, 0] * w[j][:, 1] * dw[k][:, 2]], 1) * p.inv_dx
        u = off[None, :] - fx
        vh = inter["vh"][lin]
        Cu = np.einsum("nij,nj->ni", Cbar, u)
        contrib = wt[:, None] * vbar + (c4 * wt)[:, None] * Cu
        for c in range(3):
            vh_bar[:, c] += np.bincount(lin, weights=contrib[:, c], minlength=G)
        wbar = (vbar * vh).sum(1) + c4 * (vh * Cu).sum(1)
        ubar = (c4 * wt)[:, None] * np.einsum("nji,nj->ni", Cbar, vh)
        xbar += wbar[:, None] * gw - p.inv_dx * ubar
    # grid op: the boundary, then the colliders in reverse order
    vg_bar = vh_bar * inter["gmask"]
    act = inter["act"]
    cbar = np.zeros((inter["n_colliders"], 2, 3))  # per collider: (pos_bar, lin_vel_bar)
    if inter["chain"]:
        va_bar = vg_bar[act]
        gpa = inter["gpos"][act]
        ma = inter["gm"][act] / 1e3
        for k, c, vin in reversed(inter["chain"]):
            va_bar, pb, lb = collider_vjp(p, c, gpa, vin, va_bar, mass=ma)
            cbar[k, 0] += pb
            cbar[k, 1] += lb
        vg_bar = np.zeros_like(vg_bar)
        vg_bar[act] = va_bar
    if inter["ff_chain"]:
        va_bar = vg_bar[act]
        gpa = inter["gpos"][act]
        for f, vin in reversed(inter["ff_chain"]):
            va_bar = force_field_vjp(p, f, gpa, vin, va_bar)
        vg_bar = np.zeros_like(vg_bar)
        vg_bar[act] = va_bar
    pbar = np.zeros((G, 3))
    mbar = np.zeros(G)
    pbar[act] = vg_bar[act] / inter["gm"][act][:, None]
    mbar[act] = -(vg_bar[act] * inter["gp"][act]).sum(1) / inter["gm"][act] ** 2
    # p2g scatter
    A = inter["A"]
    Abar = np.zeros((n, 3, 3))
    vbar_n = np.zeros((n, 3))
    for (i, j, k), lin in zip(_offsets(), inter["lin"]):
        off = np.array([i, j, k])
        wt = w[i][:, 0] * w[j][:, 1] * w[k][:, 2]
        gw = np.stack([dw[i][:, 0] * w[j][:, 1] * w[k][:, 2], w[i][:, 0] * dw[j][:, 1] * w[k][:, 2],
                       w[i][:, 0] * w[j][:, 1] * dw[k][:, 2]], 1) * p.inv_dx
        d = (off[None, :] - fx) * p.dx
        pb = pbar[lin]
        mb = mbar[lin]
        q = mass[:, None] * v + np.einsum("nij,nj->ni", A, d)
        wbar = mb * mass + (pb * q).sum(1)
        vbar_n += (wt * mass)[:, None] * pb
        Abar += wt[:, None, None] * pb[:, :, None] * d[:, None, :]
        xbar += wbar[:, None] * gw - wt[:, None] * np.einsum("nji,nj->ni", A, pb)
    Pbar = inter["s"] * Abar
    Cbar_n = mass[:, None, None] * Abar
    # the materials, then svd_grad (backward_svd) and compute_F_tmp.grad
    Ft, U, S, V = inter["Ft"], inter["U"], inter["S"], inter["V"]
    Ft_bar = np.zeros_like(Ft)
    Jp_bar = np.zeros(n)
    mu_bar = np.zeros(n)
    lam_bar = np.zeros(n)
    actu_bar = np.zeros(n)
    mi = np.asarray(st["mat"])
    for k, m in enumerate(mats):
        sel = mi == k
        if not sel.any():
            continue
        actu = st["actu"][sel] if st.get("actu") is not None else None
        mdir = st["mdir"][sel] if st.get("mdir") is not None else None
        ftb, ub, sb, vb, jb, mb_, lb, ab = material_vjp(m, p.eps, U[sel], S[sel], V[sel], Ft[sel], st["Jp"][sel],
                                                         mu[sel], lam[sel], actu, mdir, adj["F"][sel], adj["Jp"][sel],
                                                         Pbar[sel])
        Sd = np.zeros((int(sel.sum()), 3, 3))
        Sd[:, [0, 1, 2], [0, 1, 2]] = S[sel]
        Sbar = np.zeros_like(Sd)
        Sbar[:, [0, 1, 2], [0, 1, 2]] = sb
        Ft_bar[sel] = ftb + backward_svd(ub, Sbar, vb, U[sel], Sd, V[sel])
        Jp_bar[sel], mu_bar[sel], lam_bar[sel], actu_bar[sel] = jb, mb_, lb, ab
    F_bar_n = _mT(np.eye(3) + p.dt * C) @ Ft_bar
    Cbar_n += p.dt * Ft_bar @ _mT(F)
    out = dict(x=xbar, v=vbar_n, C=Cbar_n, F=F_bar_n, Jp=Jp_bar)
    if inter["n_colliders"]:
        out["colliders"] = cbar
    return out, mu_bar, lam_bar, actu_bar


def rollout_materials(p, mats, st0, mu, lam, n_substeps, target, grad=True, weights=None):
    """loss = |mean(x_T) - target|^2 (or, with weights [n, 3], sum(weights * x_T)) over a
    rollout of any material mix, and (grad=True) its gradients w.r.t. a uniform initial
    velocity and per-particle mu, lam."""
    states, inters = [st0], []
    st = st0
    for _ in range(n_substeps):
        st, it = forward_materials(p, mats, st, mu, lam)
        states.append(st)
        inters.append(it)
    n = st0["x"].shape[0]
    xm = states[-1]["x"].mean(0)
    if weights is None:
        loss = float(((xm - target) ** 2).sum())
        xbar = np.tile(2 * (xm - target) / n, (n, 1))
    else:
        loss = float((weights * states[-1]["x"]).sum())
        xbar = np.asarray(weights, dtype=np.float64).copy()
    if not grad:
        return loss
    adj = dict(x=xbar, v=np.zeros((n, 3)), C=np.zeros((n, 3, 3)), F=np.zeros((n, 3, 3)), Jp=np.zeros(n))
    mu_bar = np.zeros(n)
    lam_bar = np.zeros(n)
    for t in range(n_substeps - 1, -1, -1):
        adj, mb, lb, _ = backward_materials(p, mats, states[t], mu, lam, inters[t], adj)
        mu_bar += mb
        lam_bar += lb
    return loss, adj["v"].sum(0), mu_bar, lam_bar, adj


def rollout_colliders(p, mats, st0, mu, lam, colliders, lin_vel, weights, grad=True):
    """loss = sum(weights * x_T) over T = len(lin_vel) substeps of any material mix with
    kinematic colliders (tool_entity.py:178-191: pos_{t+1} = pos_t + lin_vel_t dt, a tool's
    origin kept above its floor, rot_{t+1} = exp(ang dt) rot_t), lin_vel [T, n_colliders, 3]
    the colliders' linear velocity at each substep (what set_velocity gives them), and
    (grad=True) its gradients with respect to every particle's initial velocity [n, 3], the
    colliders' initial positions [n_colliders, 3] and lin_vel [T, n_colliders, 3].  Rotations
    and angular velocities are not differentiated."""
    import dataclasses

    lin_vel = np.asarray(lin_vel, dtype=np.float64)
    T = lin_vel.shape[0]
    cols = list(colliders)
    states, inters, hist = [st0], [], []
    st = st0
    for t in range(T):
        cols = [dataclasses.replace(c, lin_vel=lin_vel[t, k].copy()) for k, c in enumerate(cols)]
        hist.append(cols)
        st, it = forward_materials(p, mats, st, mu, lam, colliders=cols)
        states.append(st)
        inters.append(it)
        cols = R.advance_colliders(p, cols)
    loss = float((weights * states[-1]["x"]).sum())
    if not grad:
        return loss
    n = st0["x"].shape[0]
    adj = dict(x=np.asarray(weights, dtype=np.float64).copy(), v=np.zeros((n, 3)), C=np.zeros((n, 3, 3)),
               F=np.zeros((n, 3, 3)), Jp=np.zeros(n))
    pos_bar = np.zeros((len(colliders), 3))  # dL/d(collider position after substep t)
    lin_bar = np.zeros_like(lin_vel)
    for t in range(T - 1, -1, -1):
        for k, c in enumerate(hist[t]):
            pb = pos_bar[k].copy()
            if c.kind == "tool" and c.pos[2] + c.lin_vel[2] * p.dt < c.floor:
                pb[2] = 0.0  # clamped to the floor: the new z depends on neither
            lin_bar[t, k] += p.dt * pb
            pos_bar[k] = pb
        adj, _, _, _ = backward_materials(p, mats, states[t], mu, lam, inters[t], adj)
        cb = adj.pop("colliders", None)
        if cb is not None:
            pos_bar += cb[:, 0]
            lin_bar[t] += cb[:, 1]
    return loss, adj["v"], pos_bar, lin_bar


# ---------------------------------------------------------------- the kernel's formulation
# The CUDA adjoint (k_adj_p2g) does not differentiate U, S, V separately: every material's
# F_new is U diag(g(s)) V^T (Liquid: J^(1/3) I) and its stress U diag(p(s)) U^T (+ the
# Muscle term), with g, p symmetric functions of the singular values s, so the adjoint of
# F_tmp follows in the SVD basis from g, p, their Jacobians and divided differences:
#   X = U^T Fn_bar V,  Z = U^T sym(P_bar) U
#   s_bar_k = sum_i X_ii dg_i/ds_k + Z_ii dp_i/ds_k + Jpn_bar dJp_new/ds_k
#   Y_ij = 1/2 [(X_ij + X_ji) (g_i - g_j)/(s_i - s_j) + (X_ij - X_ji) (g_i + g_j)/(s_i + s_j)]
#          + 2 Z_ij s_j (p_i - p_j) / (s_i^2 - s_j^2)                           (i != j)
#   F_tmp_bar = U (diag(s_bar) + Y) V^T
# The divided differences are evaluated in forms that stay exact as s_i -> s_j (through
# log(s_i / s_j) = log1p((s_i - s_j) / s_j) and expm1), so nearly equal singular values --
# the rest state and every small strain -- lose no accuracy.  Wherever the reference's
# signmax(s_j^2 - s_i^2, 1e-6) guard is inactive this equals the reference's backward; below
# it, it is the derivative that the guard approximates (tested against finite differences).
# This numpy version states the formulation in float64 for the tests.


def _ddiff_log(si, sj, ci, cj, kappa, gj):
    """(g_i - g_j) / (s_i - s_j) for g = c^kappa-type maps: g_i - g_j = g_j expm1(kappa log(c_i / c_j)),
    with c the clamped magnitude of s (its derivative 1/s where unclamped)."""
    den = si - sj
    L = np.log1p((ci - cj) / cj)
    with np.errstate(invalid="ignore", divide="ignore"):
        dd = gj * np.expm1(kappa * L) / np.where(den != 0, den, 1.0)
    lim = gj * kappa / sj
    return np.where(den != 0, dd, np.where(ci == np.abs(si), lim, 0.0))


def material_spectral(mat, eps, s, Jp, mu, lam):
    """g, p and the derivatives the spectral adjoint needs, per particle (float64 numpy)."""
    n = s.shape[0]
    Jk = np.stack([s[:, 1] * s[:, 2], s[:, 0] * s[:, 2], s[:, 0] * s[:, 1]], 1)
    J = s[:, 0] * Jk[:, 0]
    I3 = np.eye(3)
    o = dict(ident=np.zeros(n, bool), liquid=False, Dg=np.zeros((n, 3, 3)), DDg=np.zeros((n, 3, 3)),
             g=np.zeros((n, 3)), dg_dJp=np.zeros((n, 3)), dg_dmu=np.zeros((n, 3)), dg_dlam=np.zeros((n, 3)),
             dJpn_ds=np.zeros((n, 3)), dJpn_dJp=np.ones(n), dp_dJp=np.zeros((n, 3)))
    k = mat.kind

    def corot(g, Dg, DDg, muc, lamc):
        p = 2 * muc[:, None] * (g - 1) * g + (lamc * J * (J - 1))[:, None]
        Dp = 2 * muc[:, None, None] * (2 * g - 1)[:, :, None] * Dg + (lamc * (2 * J - 1))[:, None, None] * Jk[:, None, :]
        DDp = 2 * muc[:, None, None] * (g[:, :, None] + g[:, None, :] - 1) * DDg
        return p, Dp, DDp, 2 * (g - 1) * g, np.broadcast_to((J * (J - 1))[:, None], (n, 3))

    def ident():
        o["ident"][:] = True
        o["g"] = s.copy()
        o["Dg"] = np.broadcast_to(I3, (n, 3, 3)).copy()
        o["DDg"] = np.ones((n, 3, 3))

    if k == R.KIND_ELASTIC and mat.neohookean:
        ident()
        p = mu[:, None] * s * s + (lam * np.log(J) - mu)[:, None]
        Dp = 2 * mu[:, None, None] * s[:, :, None] * I3 + (lam / J)[:, None, None] * Jk[:, None, :]
        DDp = mu[:, None, None] * (s[:, :, None] + s[:, None, :])
        dpm, dpl = s * s - 1, np.broadcast_to(np.log(J)[:, None], (n, 3))
    elif k == R.KIND_ELASTIC or k == R.KIND_LIQUID:
        if k == R.KIND_LIQUID:
            o["liquid"] = True
            o["J"], o["Jk"] = J, Jk
        else:
            ident()
        p, Dp, DDp, dpm, dpl = corot(s, np.broadcast_to(I3, (n, 3, 3)), np.ones((n, 3, 3)), mu, lam)
    elif k == R.KIND_ELASTOPLASTIC and mat.use_von_mises:
        Sc = np.maximum(s, 0.05)
        de = np.where(s > 0.05, 1.0 / s, 0.0)
        e = np.log(Sc)
        eh = e - e.mean(1, keepdims=True)
        nn = np.sqrt((eh * eh).sum(1) + eps)
        tau = mat.von_mises_yield_stress / (2 * mu)
        y = nn - tau > 0
        r = tau / nn
        g_y = np.exp(e.mean(1, keepdims=True) + r[:, None] * eh)
        dedk = 1 / 3 + r[:, None, None] * (I3 - 1 / 3) - (r / nn**2)[:, None, None] * eh[:, :, None] * eh[:, None, :]
        Dg_y = g_y[:, :, None] * dedk * de[:, None, :]
        DDg_y = _ddiff_log(s[:, :, None], s[:, None, :], Sc[:, :, None], Sc[:, None, :], r[:, None, None],
                           g_y[:, None, :])
        dgmu_y = -g_y * eh * (tau / (nn * mu))[:, None]
        g = np.where(y[:, None], g_y, s)
        Dg = np.where(y[:, None, None], Dg_y, I3)
        DDg = np.where(y[:, None, None], DDg_y, 1.0)
        o["ident"] = ~y
        o.update(g=g, Dg=Dg, DDg=DDg, dg_dmu=np.where(y[:, None], dgmu_y, 0.0))
        p, Dp, DDp, dpm, dpl = corot(g, Dg, DDg, mu, lam)
        dpm = dpm + 2 * mu[:, None] * (2 * g - 1) * o["dg_dmu"]
    elif k == R.KIND_ELASTOPLASTIC or k == R.KIND_SNOW:
        lo, hi = 1 - mat.yield_lower, 1 + mat.yield_higher
        g = np.clip(s, lo, hi)
        free = (s > lo) & (s < hi)
        Dg = free[:, :, None] * I3
        den = s[:, :, None] - s[:, None, :]
        with np.errstate(invalid="ignore", divide="ignore"):
            DDg = np.where(den != 0, (g[:, :, None] - g[:, None, :]) / np.where(den != 0, den, 1), free[:, :, None] * 1.0)
        o.update(g=g, Dg=Dg, DDg=DDg)
        if k == R.KIND_SNOW:
            h = np.exp(10 * (1.0 - Jp))
            Jpn = Jp * (s / g).prod(1)
            o["dJpn_ds"] = np.where(free, 0.0, Jpn[:, None] / s)
            o["dJpn_dJp"] = (s / g).prod(1)
            p, Dp, DDp, dpm, dpl = corot(g, Dg, DDg, mu * h, lam * h)
            o["dp_dJp"] = -10 * p
            dpm, dpl = dpm * h[:, None], dpl * h[:, None]
        else:
            p, Dp, DDp, dpm, dpl = corot(g, Dg, DDg, mu, lam)
    else:  # sand
        Sc = np.maximum(np.abs(s), 1e-4)
        de = np.where(np.abs(s) > 1e-4, 1.0 / s, 0.0)
        e = np.log(Sc)
        tr = e.sum(1) + Jp
        eh = e - (tr / 3)[:, None]
        nn = np.sqrt((eh * eh).sum(1) + eps)
        c1 = (3 * lam + 2 * mu) / (2 * mu)
        q = c1 * mat.alpha
        dg = nn + q * tr
        expand = tr >= 0
        y = (~expand) & (dg > 0)
        kap = np.where(y, -q * tr / nn, 1.0)
        ls = np.where(expand[:, None], 0.0, np.where(y[:, None], (tr / 3)[:, None] + kap[:, None] * eh, e))
        dls_de_y = 1 / 3 - q[:, None, None] * (eh[:, :, None] / nn[:, None, None] + (tr / nn)[:, None, None] * (I3 - 1 / 3)
                                              - (tr / nn**3)[:, None, None] * eh[:, :, None] * (eh + (Jp / 3)[:, None])[:, None, :])
        dls_dJp_y = 1 / 3 - q[:, None] * (eh / nn[:, None] - (tr / (3 * nn))[:, None]
                                         - (tr * Jp / (3 * nn**3))[:, None] * eh)
        dls_dq_y = -(tr / nn)[:, None] * eh
        dls_de = np.where(expand[:, None, None], 0.0, np.where(y[:, None, None], dls_de_y, I3))
        dls_dJp = np.where(y[:, None], dls_dJp_y, 0.0)
        dls_dq = np.where(y[:, None], dls_dq_y, 0.0)
        g = np.exp(ls)
        Dls = dls_de * de[:, None, :]
        dq_dmu = mat.alpha * (-3 * lam / (2 * mu * mu))
        dq_dlam = mat.alpha * 3 / (2 * mu)
        DDg = np.where(expand[:, None, None], 0.0,
                       _ddiff_log(s[:, :, None], s[:, None, :], Sc[:, :, None], Sc[:, None, :], kap[:, None, None],
                                  g[:, None, :]))
        o.update(g=g, Dg=g[:, :, None] * Dls, DDg=DDg, dg_dJp=g * dls_dJp,
                 dg_dmu=g * dls_dq * dq_dmu[:, None], dg_dlam=g * dls_dq * dq_dlam[:, None])
        o["dJpn_ds"] = np.where(expand[:, None], de, 0.0)
        o["dJpn_dJp"] = np.where(expand, 1.0, 0.0)
        p = 2 * mu[:, None] * ls + (lam * ls.sum(1))[:, None]
        Dp = 2 * mu[:, None, None] * Dls + lam[:, None, None] * Dls.sum(1)[:, None, :]
        o["dp_dJp"] = 2 * mu[:, None] * dls_dJp + (lam * dls_dJp.sum(1))[:, None]
        dlsq = 2 * mu[:, None] * dls_dq + (lam * dls_dq.sum(1))[:, None]
        dpm = 2 * ls + dlsq * dq_dmu[:, None]
        dpl = np.broadcast_to(ls.sum(1)[:, None], (n, 3)) + dlsq * dq_dlam[:, None]
        # (p_i - p_j) / (s_i - s_j) = 2 mu kap log(c_i / c_j) / (s_i - s_j)
        den = s[:, :, None] - s[:, None, :]
        L = np.log1p((Sc[:, :, None] - Sc[:, None, :]) / Sc[:, None, :])
        with np.errstate(invalid="ignore", divide="ignore"):
            DDp = np.where(den != 0, 2 * mu[:, None, None] * kap[:, None, None] * L / np.where(den != 0, den, 1),
                           2 * mu[:, None, None] * kap[:, None, None] / s[:, None, :])
        DDp = np.where(expand[:, None, None], 0.0, DDp)
    o.update(p=p, Dp=Dp, DDp=DDp, dp_dmu=dpm, dp_dlam=dpl)
    return o


def material_vjp_spectral(mat, eps, U, S, V, Ft, Jp, mu, lam, Fn_bar, Jpn_bar, P_bar):
    """The kernel's adjoint of one material (without the Muscle term): returns F_tmp_bar,
    Jp_bar, mu_bar, lam_bar."""
    s = S
    o = material_spectral(mat, eps, s, Jp, mu, lam)
    X = _mT(U) @ Fn_bar @ V
    Z = _mT(U) @ (0.5 * (P_bar + _mT(P_bar))) @ U
    Xd = np.diagonal(X, axis1=1, axis2=2)
    Zd = np.diagonal(Z, axis1=1, axis2=2)
    use_x = ~(o["ident"] | o["liquid"])
    sbar = np.einsum("ni,nik->nk", Zd, o["Dp"]) + Jpn_bar[:, None] * o["dJpn_ds"]
    sbar += np.where(use_x[:, None], np.einsum("ni,nik->nk", Xd, o["Dg"]), 0.0)
    Jpb = Jpn_bar * o["dJpn_dJp"] + (Zd * o["dp_dJp"]).sum(1) + np.where(use_x, (Xd * o["dg_dJp"]).sum(1), 0.0)
    mub = (Zd * o["dp_dmu"]).sum(1) + np.where(use_x, (Xd * o["dg_dmu"]).sum(1), 0.0)
    lamb = (Zd * o["dp_dlam"]).sum(1) + np.where(use_x, (Xd * o["dg_dlam"]).sum(1), 0.0)
    ss = s[:, :, None] + s[:, None, :]
    with np.errstate(invalid="ignore", divide="ignore"):
        G = np.where(np.abs(ss) > 1e-12, (o["g"][:, :, None] + o["g"][:, None, :]) / np.where(np.abs(ss) > 1e-12, ss, 1), 0)
        Gam = np.where(np.abs(ss) > 1e-12, o["DDp"] / np.where(np.abs(ss) > 1e-12, ss, 1), 0)
    Y = 2 * Z * s[:, None, :] * Gam
    Y += np.where(use_x[:, None, None], 0.5 * ((X + _mT(X)) * o["DDg"] + (X - _mT(X)) * G), 0.0)
    if o["liquid"]:
        c = np.cbrt(o["J"])
        Jb = np.trace(Fn_bar, axis1=1, axis2=2) * c / (3 * o["J"])
        sbar += Jb[:, None] * o["Jk"]
    idx = np.arange(3)
    Y[:, idx, idx] = sbar
    Ftb = U @ Y @ _mT(V)
    Ftb += np.where(o["ident"][:, None, None], Fn_bar, 0.0)
    return Ftb, Jpb, mub, lamb
