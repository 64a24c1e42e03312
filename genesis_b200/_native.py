"""ctypes binding of the C ABI declared in include/genesis_b200_mpm.h.

The shared library ``libgenesis_b200_mpm.so`` is built in-tree (see
``genesis_b200.build``).  There is no fallback: if the library is missing, every
entry point raises ``NativeLibraryError``.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

LIB_NAME = "libgenesis_b200_mpm.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

ABI_VERSION = 14

MPM_OK = 0
MPM_E_INVALID = -1
MPM_E_CUDA = -2
MPM_E_CAPACITY = -3
MPM_E_NOT_SORTED = -4
ERROR_NAMES = {
    MPM_E_INVALID: "invalid argument",
    MPM_E_CUDA: "CUDA runtime error",
    MPM_E_CAPACITY: "size exceeds a compiled-in limit",
    MPM_E_NOT_SORTED: "particles were never sorted",
}

MPM_STATUS_NAN = 1
MPM_STATUS_OUT_OF_GRID = 2
MPM_STATUS_NONFINITE_VEL = 4

NOALLOC_SCRATCH_BYTES = 32 << 20

MPM_STATE_CH = 25
CH_X, CH_V, CH_C, CH_F, CH_JP = 0, 3, 6, 15, 24
MPM_BLOCK = 4
PFLAG_ACTIVE = 1
PFLAG_FREE = 2
PROBF_NONFREE = 1
PROBF_CPIC = 2

MAT_ELASTIC, MAT_ELASTOPLASTIC, MAT_LIQUID, MAT_SAND, MAT_SNOW = 0, 1, 2, 3, 4

# kernel kinds of mpm_substeps_profile
KIND_NAMES = ("sort", "p2g", "grid_op", "g2p", "g2p2g")
MATF_NEOHOOKEAN = 1
MATF_VON_MISES = 2
MATF_MUSCLE = 4


class NativeLibraryError(RuntimeError):
    pass


class MPMNativeError(RuntimeError):
    def __init__(self, fn: str, rc: int):
        super().__init__(f"{fn} failed: {ERROR_NAMES.get(rc, 'error')} (rc={rc})")
        self.rc = rc


class Instance(C.Structure):
    _fields_ = [
        ("p_begin", C.c_int32),
        ("p_count", C.c_int32),
        ("res", C.c_int32 * 3),
        ("nblk", C.c_int32 * 3),
        ("lower_cell", C.c_int32 * 3),
        ("mat_base", C.c_int32),
        ("blk_base", C.c_int64),
        ("dx", C.c_float),
        ("inv_dx", C.c_float),
        ("dt", C.c_float),
        ("eps", C.c_float),
        ("gravity", C.c_float * 3),
        ("bnd_lo", C.c_float * 3),
        ("bnd_hi", C.c_float * 3),
        ("stress_scale", C.c_float),
        ("c_scale", C.c_float),
        ("pad0", C.c_float),
    ]


class Material(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("flags", C.c_int32),
        ("mu", C.c_float),
        ("lam", C.c_float),
        ("mass", C.c_float),
        ("default_Jp", C.c_float),
        ("clamp_lo", C.c_float),
        ("clamp_hi", C.c_float),
        ("vm_threshold", C.c_float),
        ("sand_c1", C.c_float),
        ("sand_alpha", C.c_float),
        ("muscle_stiffness", C.c_float),
    ]


class Problem(C.Structure):
    _fields_ = [
        ("n_instances", C.c_int32),
        ("n_particles", C.c_int32),
        ("n_blocks", C.c_int64),
        ("n_materials", C.c_int32),
        ("chunk_particles", C.c_int32),
        ("max_chunks", C.c_int32),
        ("grid_ctas", C.c_int32),
        ("flags", C.c_int32),
    ]


class Particles(C.Structure):
    _fields_ = [
        ("state", C.c_void_p),
        ("state_stride", C.c_int64),
        ("mat", C.c_void_p),
        ("pflags", C.c_void_p),
        ("gid", C.c_void_p),
        ("slot", C.c_void_p),
        ("mu_p", C.c_void_p),
        ("lam_p", C.c_void_p),
        ("actu", C.c_void_p),
        ("muscle_dir", C.c_void_p),
        ("cpic_normal", C.c_void_p),
        ("cpic_sep", C.c_void_p),
    ]


class Tables(C.Structure):
    _fields_ = [
        ("instances", C.c_void_p),
        ("materials", C.c_void_p),
        ("colliders", C.c_void_p),
        ("n_colliders", C.c_int32),
        ("pad0", C.c_int32),
        ("collider_force", C.c_void_p),
        ("sdf_voxels", C.c_void_p),
        ("force_fields", C.c_void_p),
        ("n_force_fields", C.c_int32),
        ("pad1", C.c_int32),
        ("ff_perm", C.c_void_p),
    ]


class ForceField(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("active", C.c_int32),
        ("vec", C.c_float * 3),
        ("dir", C.c_float * 3),
        ("center", C.c_float * 3),
        ("strength", C.c_float),
        ("strength2", C.c_float),
        ("radius", C.c_float),
        ("falloff_pow", C.c_float),
        ("falloff_min", C.c_float),
        ("falloff_max", C.c_float),
        ("flow", C.c_float),
        ("damping", C.c_float),
        ("linear", C.c_float),
        ("quadratic", C.c_float),
        ("frequency", C.c_float),
        ("perm_offset", C.c_int32),
        ("seed", C.c_uint32),
    ]


FF_CONSTANT, FF_WIND, FF_POINT, FF_DRAG, FF_NOISE, FF_VORTEX, FF_TURBULENCE = range(7)


COLLIDER_SPHERE, COLLIDER_PLANE, COLLIDER_BOX, COLLIDER_TOOL, COLLIDER_SDF = 0, 1, 2, 3, 4


class Collider(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("instance", C.c_int32),
        ("pos", C.c_float * 3),
        ("rot", C.c_float * 9),
        ("data", C.c_float * 3),
        ("lin_vel", C.c_float * 3),
        ("ang_vel", C.c_float * 3),
        ("friction", C.c_float),
        ("softness", C.c_float),
        ("restitution", C.c_float),
        ("sdf_res", C.c_int32),
        ("sdf_pad", C.c_int32),
        ("sdf_offset", C.c_int64),
        ("sdf_scale", C.c_float * 3),
        ("floor", C.c_float),
        ("sdf_res3", C.c_int32 * 3),
        ("sdf_cell", C.c_float),
        ("sdf_max", C.c_float),
        ("sdf_pad2", C.c_float),
    ]


_P = C.POINTER
vp = C.c_void_p
i32 = C.c_int32
i64 = C.c_int64

# name -> (restype, argtypes)
SIGNATURES = {
    "mpm_abi_version": (C.c_int, []),
    "mpm_struct_sizes": (C.c_int, [_P(C.c_int32)]),
    "mpm_max_chunks": (C.c_int, [i32, i64, i32, _P(C.c_int32)]),
    "mpm_workspace_bytes": (C.c_int, [_P(Problem), _P(C.c_uint64)]),
    "mpm_workspace_init": (C.c_int, [_P(Problem), vp, vp]),
    "mpm_grid_offsets": (C.c_int, [_P(Problem), _P(C.c_uint64), _P(C.c_uint64)]),
    "mpm_sort_particles": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), vp, vp]),
    "mpm_p2g": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), vp, vp]),
    "mpm_grid_op": (C.c_int, [_P(Problem), _P(Tables), vp, vp]),
    "mpm_g2p": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), vp, vp]),
    "mpm_g2p2g": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), vp, vp]),
    "mpm_substeps": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), vp, i32, i32, i64, vp]),
    "mpm_substeps_noalloc": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), i32, i32, i64, vp]),
    "mpm_noalloc_status": (C.c_int, [_P(Problem), i32, _P(C.c_uint32), vp, vp]),
    "mpm_substeps_profile": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), vp, i32, i32, i64, vp, vp, vp]),
    "mpm_adjoint_workspace_bytes": (C.c_int, [_P(Problem), _P(C.c_uint64)]),
    "mpm_substep_adjoint": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), vp, vp, vp, vp, vp]),
    "mpm_substep_adjoint_colliders": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), vp, vp, vp, vp, vp, vp]),
    "mpm_record_grid_bytes": (C.c_int, [_P(Problem), _P(C.c_uint64)]),
    "mpm_substeps_record": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), vp, i32, vp, vp, vp]),
    "mpm_substeps_adjoint_recorded": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), i32, i32, vp, vp, vp, vp, vp,
                                                vp]),
    "mpm_status": (C.c_int, [_P(Problem), vp, i32, _P(C.c_uint32), vp]),
    "mpm_status_enqueue": (C.c_int, [_P(Problem), vp, vp, vp]),
    "mpm_fallback_count": (C.c_int, [_P(Problem), vp, i32, _P(C.c_uint64), vp]),
    "mpm_instance_status": (C.c_int, [_P(Problem), vp, i32, vp, vp]),
    "mpm_instance_status_enqueue": (C.c_int, [_P(Problem), vp, i32, vp, vp]),
    "mpm_get_state": (C.c_int, [_P(Problem), _P(Particles), vp, vp, vp, vp, vp, vp, vp]),
    "mpm_set_state": (C.c_int, [_P(Problem), _P(Particles), vp, vp, vp, vp, vp, vp, vp]),
    "mpm_set_particles_pos": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), i32, vp, vp, vp]),
    "mpm_set_particles_vel": (C.c_int, [_P(Problem), _P(Particles), i32, vp, vp, vp]),
    "mpm_set_particles_active": (C.c_int, [_P(Problem), _P(Particles), i32, vp, vp, vp]),
    "mpm_set_particles_free": (C.c_int, [_P(Problem), _P(Particles), i32, vp, vp, vp]),
    "mpm_update_render_fields": (C.c_int, [_P(Problem), _P(Particles), i32, i32, vp, vp, vp, i32, i32, vp, vp, vp,
                                           vp, vp]),
    "mpm_sdf_voxelize": (C.c_int, [vp, i32, vp, i32, i32, C.c_float, vp, vp]),
    "mpm_sdf_grid": (C.c_int, [vp, i32, vp, i32, _P(C.c_float), _P(C.c_float), _P(C.c_int32), vp, vp]),
    "mpm_graph_create": (C.c_int, [_P(Problem), _P(Tables), _P(Particles), vp, i32, i32, i64, vp, _P(vp)]),
    "mpm_graph_launch": (C.c_int, [vp, vp]),
    "mpm_graph_destroy": (C.c_int, [vp]),
}

_lib = None
_lock = threading.Lock()


def load(path: str | None = None):
    """Load the shared library (once) and bind every entry point.  Raises if absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or os.environ.get("GENESIS_B200_LIB") or LIB_PATH
        if not os.path.exists(p):
            raise NativeLibraryError(
                f"{LIB_NAME} not found at {p}; build it with `python -c 'import genesis_b200.build as b; b.build()'`"
            )
        lib = C.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if lib.mpm_abi_version() != ABI_VERSION:
            raise NativeLibraryError("ABI version mismatch between genesis_b200 and " + LIB_NAME)
        sizes = (C.c_int32 * 7)()
        lib.mpm_struct_sizes(sizes)
        mine = (C.sizeof(Instance), C.sizeof(Material), C.sizeof(Problem), C.sizeof(Particles), C.sizeof(Tables),
                C.sizeof(Collider), C.sizeof(ForceField))
        if tuple(sizes) != mine:
            raise NativeLibraryError(f"struct layout mismatch: library {tuple(sizes)} vs binding {mine}")
        _lib = lib
        return lib


def check(fn: str, rc: int):
    if rc != MPM_OK:
        raise MPMNativeError(fn, rc)


def call(name: str, *args):
    lib = load()
    rc = getattr(lib, name)(*args)
    check(name, rc)
    return rc


def instances_to_bytes(insts: list[Instance]) -> np.ndarray:
    arr = (Instance * len(insts))(*insts)
    return np.frombuffer(bytes(arr), dtype=np.uint8).copy()


def materials_to_bytes(mats: list[Material]) -> np.ndarray:
    arr = (Material * len(mats))(*mats)
    return np.frombuffer(bytes(arr), dtype=np.uint8).copy()
