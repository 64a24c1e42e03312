"""ctypes driver of the C/OpenMP restatement (oracle/mpm_ref.c) -- TEST INFRASTRUCTURE ONLY.

Builds oracle/_build/libmpm_ref_{f32,f64}.so with gcc on first use (no CUDA needed).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import mpm_ref as R

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")


def build(force: bool = False):
    outs = [os.path.join(BUILD, f"libmpm_ref_{t}.so") for t in ("f32", "f64")]
    src = os.path.join(HERE, "mpm_ref.c")
    if force or not all(os.path.exists(o) and os.path.getmtime(o) >= os.path.getmtime(src) for o in outs):
        subprocess.run(["make", "-C", HERE, "-B" if force else "all"], check=True, capture_output=True)
    return outs


def _real(dtype):
    return C.c_float if np.dtype(dtype) == np.float32 else C.c_double


def _structs(dtype):
    Rt = _real(dtype)

    class Params(C.Structure):
        _fields_ = [
            ("res", C.c_int32 * 3),
            ("lower_cell", C.c_int32 * 3),
            ("dx", Rt), ("inv_dx", Rt), ("dt", Rt), ("eps", Rt),
            ("gravity", Rt * 3), ("bnd_lo", Rt * 3), ("bnd_hi", Rt * 3),
            ("stress_scale", Rt), ("c_scale", Rt),
        ]

    class Mat(C.Structure):
        _fields_ = [
            ("kind", C.c_int32), ("flags", C.c_int32),
            ("mu", Rt), ("lam", Rt), ("mass", Rt),
            ("clamp_lo", Rt), ("clamp_hi", Rt), ("vm_threshold", Rt), ("sand_c1", Rt), ("sand_alpha", Rt),
            ("muscle_stiffness", Rt),
        ]

    class Coll(C.Structure):
        _fields_ = [
            ("kind", C.c_int32),
            ("pos", Rt * 3), ("rot", Rt * 9), ("data", Rt * 3), ("lin_vel", Rt * 3), ("ang_vel", Rt * 3),
            ("friction", Rt), ("softness", Rt), ("restitution", Rt),
            ("sdf", C.c_void_p), ("sdf_res", C.c_int32), ("sdf_scale", Rt * 3), ("floor", Rt),
            ("sdf_res3", C.c_int32 * 3), ("sdf_cell", Rt), ("sdf_max", Rt),
        ]

    return Params, Mat, Coll


_libs = {}


def lib(dtype):
    key = np.dtype(dtype).name
    if key not in _libs:
        build()
        path = os.path.join(BUILD, "libmpm_ref_f32.so" if key == "float32" else "libmpm_ref_f64.so")
        L = C.CDLL(path)
        L.ref_substeps.restype = C.c_int
        L.ref_substeps_lame.restype = C.c_int
        L.ref_substeps_ext.restype = C.c_int
        L.ref_substeps_full.restype = C.c_int
        L.ref_substeps_cpic.restype = C.c_int
        L.ref_max_threads.restype = C.c_int
        _libs[key] = L
    return _libs[key]


def max_threads() -> int:
    return int(lib(np.float64).ref_max_threads())


def substeps(p: R.Params, mats: list[R.Material], st: dict, n_substeps: int, n_threads: int = 0,
             mu_p=None, lam_p=None, branch_margin=None) -> tuple[dict, int]:
    """Run n_substeps in C on a copy of the state; returns (new_state, status).  mu_p/lam_p:
    optional per-particle Lame parameters.  branch_margin: optional float array [n] of the
    state's dtype, lowered in place to each particle's smallest distance (over the run) to
    its return mapping's branch switch (Sand |tr|, von Mises |delta_gamma|, clamp distance);
    initialise it to +inf."""
    if branch_margin is not None:
        L = lib(p.dtype)
        assert branch_margin.dtype == np.dtype(p.dtype) and branch_margin.flags.c_contiguous
        L.ref_set_branch_margin(branch_margin.ctypes.data_as(C.c_void_p))
        try:
            return substeps(p, mats, st, n_substeps, n_threads, mu_p, lam_p)
        finally:
            L.ref_set_branch_margin(None)
    dt = np.dtype(p.dtype)
    L = lib(dt)
    Params, Mat, Coll = _structs(dt)
    P = Params()
    for d in range(3):
        P.res[d] = int(p.grid_res[d])
        P.lower_cell[d] = int(p.lower_cell[d])
        P.gravity[d] = float(p.gravity[d])
        P.bnd_lo[d] = float(p.bnd_lo[d])
        P.bnd_hi[d] = float(p.bnd_hi[d])
    P.dx, P.inv_dx, P.dt, P.eps = p.dx, p.inv_dx, p.dt, p.eps
    P.stress_scale = -p.dt * p.p_vol * 4 * p.inv_dx * p.inv_dx
    P.c_scale = 4 * p.inv_dx
    marr = (Mat * len(mats))()
    for i, m in enumerate(mats):
        flags = (1 if (m.kind == R.KIND_ELASTIC and m.neohookean) else 0) | (
            2 if (m.kind == R.KIND_ELASTOPLASTIC and m.use_von_mises) else 0) | (4 if m.muscle else 0)
        marr[i].kind = m.kind
        marr[i].flags = flags
        marr[i].mu, marr[i].lam = m.mu, m.lam
        marr[i].mass = R.particle_mass(p, m)
        marr[i].clamp_lo, marr[i].clamp_hi = 1 - m.yield_lower, 1 + m.yield_higher
        marr[i].vm_threshold = m.von_mises_yield_stress / (2 * m.mu) if m.mu else 0.0
        marr[i].sand_c1 = (3 * m.lam + 2 * m.mu) / (2 * m.mu) if m.mu else 0.0
        marr[i].sand_alpha = m.alpha
        marr[i].muscle_stiffness = m.stiffness if m.muscle else 0.0
    n = st["x"].shape[0]
    x = np.ascontiguousarray(st["x"], dtype=dt).copy()
    v = np.ascontiguousarray(st["v"], dtype=dt).copy()
    Cm = np.ascontiguousarray(st["C"], dtype=dt).reshape(n, 9).copy()
    F = np.ascontiguousarray(st["F"], dtype=dt).reshape(n, 9).copy()
    Jp = np.ascontiguousarray(st["Jp"], dtype=dt).copy()
    mat = np.ascontiguousarray(st["mat"], dtype=np.int32)
    act = np.ascontiguousarray(st["active"], dtype=np.uint8)
    G = int(np.prod(p.grid_res))
    grid = np.zeros(4 * G, dtype=dt)
    gvel = np.zeros(3 * G, dtype=dt)
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    if st.get("colliders"):
        cs = st["colliders"]
        carr = (Coll * len(cs))()
        kinds = {"sphere": 0, "plane": 1, "box": 2, "tool": 3, "sdf": 4}
        keep = []  # the tools' voxel arrays stay alive for the call
        for i, c in enumerate(cs):
            carr[i].kind = kinds[c.kind]
            if c.kind == "sdf":
                vox = np.ascontiguousarray(np.concatenate([np.asarray(c.sdf, dtype=dt).reshape(-1),
                                                           np.asarray(c.sdf_grad, dtype=dt).reshape(-1)]))
                keep.append(vox)
                carr[i].sdf = vox.ctypes.data_as(C.c_void_p)
                for d in range(3):
                    carr[i].sdf_res3[d] = int(np.shape(c.sdf)[d])
                    carr[i].sdf_scale[d] = float(c.sdf_scale[d])
                carr[i].sdf_cell = float(c.sdf_cell)
                carr[i].sdf_max = float(c.sdf_max)
            if c.kind == "tool":
                vox = np.ascontiguousarray(c.sdf, dtype=dt).reshape(-1)
                keep.append(vox)
                carr[i].sdf = vox.ctypes.data_as(C.c_void_p)
                carr[i].sdf_res = int(round(len(vox) ** (1 / 3)))
                for d in range(3):
                    carr[i].sdf_scale[d] = float(np.broadcast_to(c.sdf_scale, (3,))[d])
                carr[i].floor = float(c.floor)
            for d in range(3):
                carr[i].pos[d] = c.pos[d]
                carr[i].data[d] = c.data[d]
                carr[i].lin_vel[d] = c.lin_vel[d]
                carr[i].ang_vel[d] = c.ang_vel[d]
            for k in range(9):
                carr[i].rot[k] = np.asarray(c.rot, dtype=np.float64).reshape(9)[k]
            carr[i].friction, carr[i].softness, carr[i].restitution = c.friction, c.softness, c.restitution
        forces = np.zeros((len(cs), 6), dtype=dt)
        actu = np.ascontiguousarray(st["actu"], dtype=dt) if st.get("actu") is not None else None
        mdir = np.ascontiguousarray(st["mdir"], dtype=dt).reshape(n, 3) if st.get("mdir") is not None else None
        mu_a = np.ascontiguousarray(mu_p, dtype=dt) if mu_p is not None else None
        lam_a = np.ascontiguousarray(lam_p, dtype=dt) if lam_p is not None else None
        opt = lambda a: ptr(a) if a is not None else None
        # CPIC: st["cpic_normal"] [n_colliders, n, 3] (zeros at the start) switches it on
        rn = st.get("cpic_normal")
        rn = np.ascontiguousarray(rn, dtype=dt).copy() if rn is not None else None
        rc = L.ref_substeps_cpic(C.byref(P), marr, n, ptr(x), ptr(v), ptr(Cm), ptr(F), ptr(Jp), ptr(mat), ptr(act),
                                 int(n_substeps), ptr(grid), ptr(gvel), int(n_threads), opt(mu_a), opt(lam_a),
                                 opt(actu), opt(mdir), carr, len(cs), ptr(forces), opt(rn))
        moved = []
        for i, c in enumerate(cs):
            moved.append(R.Collider(c.kind, np.array(carr[i].pos[:]), np.array(carr[i].rot[:]).reshape(3, 3),
                                    np.asarray(c.data), np.asarray(c.lin_vel), np.asarray(c.ang_vel), c.friction,
                                    c.softness, c.restitution, c.sdf, c.sdf_scale, c.floor, c.sdf_grad, c.sdf_cell,
                                    c.sdf_max))
        out = dict(st)
        out.update(x=x, v=v, C=Cm.reshape(n, 3, 3), F=F.reshape(n, 3, 3), Jp=Jp, colliders=moved, forces=forces)
        if rn is not None:
            out["cpic_normal"] = rn
        return out, int(rc)
    if st.get("actu") is not None:
        actu = np.ascontiguousarray(st["actu"], dtype=dt)
        mdir = np.ascontiguousarray(st["mdir"], dtype=dt).reshape(n, 3)
        mu_a = np.ascontiguousarray(mu_p, dtype=dt) if mu_p is not None else None
        lam_a = np.ascontiguousarray(lam_p, dtype=dt) if lam_p is not None else None
        rc = L.ref_substeps_ext(C.byref(P), marr, n, ptr(x), ptr(v), ptr(Cm), ptr(F), ptr(Jp), ptr(mat), ptr(act),
                                int(n_substeps), ptr(grid), ptr(gvel), int(n_threads),
                                ptr(mu_a) if mu_a is not None else None, ptr(lam_a) if lam_a is not None else None,
                                ptr(actu), ptr(mdir))
    elif mu_p is not None:
        mu_a = np.ascontiguousarray(mu_p, dtype=dt)
        lam_a = np.ascontiguousarray(lam_p, dtype=dt)
        rc = L.ref_substeps_lame(C.byref(P), marr, n, ptr(x), ptr(v), ptr(Cm), ptr(F), ptr(Jp), ptr(mat), ptr(act),
                                 int(n_substeps), ptr(grid), ptr(gvel), int(n_threads), ptr(mu_a), ptr(lam_a))
    else:
        rc = L.ref_substeps(C.byref(P), marr, n, ptr(x), ptr(v), ptr(Cm), ptr(F), ptr(Jp), ptr(mat), ptr(act),
                            int(n_substeps), ptr(grid), ptr(gvel), int(n_threads))
    out = dict(st)
    out.update(x=x, v=v, C=Cm.reshape(n, 3, 3), F=F.reshape(n, 3, 3), Jp=Jp)
    return out, int(rc)
