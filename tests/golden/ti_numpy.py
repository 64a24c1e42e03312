"""A numpy stand-in for the subset of gstaichi that Genesis's MPM path uses, and a loader
that runs the reference's own MPM source files on it.

TEST INFRASTRUCTURE ONLY (fixture generation).  gstaichi (the reference's kernel language,
``gstaichi==4.5.0``, pyproject.toml:13) is not installed here, but the reference's MPM
kernels are plain Python bodies under ``@ti.kernel`` / ``@ti.func``.  With this module
standing in for ``gstaichi`` and small stubs standing in for the rest of the ``genesis``
package, the reference files below are imported UNCHANGED from the reference checkout and
their kernels run as serial Python loops over numpy values:

  genesis/engine/solvers/base_solver.py        Solver (dt, substep_dt, gravity)
  genesis/engine/solvers/mpm_solver.py         MPMSolver: __init__, fields, _kernel_add_particles,
                                               reset_grid_and_grad, compute_F_tmp, svd, p2g, g2p,
                                               copy_frame, _is_state_valid, backward_svd, signmax
  genesis/engine/couplers/legacy_coupler.py    LegacyCoupler.mpm_grid_op, preprocess
  genesis/engine/boundaries/boundaries.py      CubeBoundary
  genesis/engine/materials/base.py             Material
  genesis/engine/materials/MPM/*.py            Base, Elastic, ElastoPlastic, Liquid, Muscle, Sand, Snow

Semantics emulated (as Taichi defines them):
  * scalars and vectors/matrices are values: ``@ti.func`` arguments are copied on entry
    (pass by value), and reading a field element yields a copy that writes back only on
    item assignment (``field[i].pos[d] = x``) or attribute assignment;
  * ``@ti.kernel`` arguments annotated ``ti.f32`` are rounded to float32, ``ti.i32`` to int;
  * ``Matrix.norm(eps)`` = sqrt(sum of squares + eps); ``determinant`` is the 3x3 cofactor
    expansion; ``ti.max``/``ti.min`` are element-wise;
  * loops run serially in index order (the reference's CPU backend with one thread).
The one substitution: ``ti.svd`` is gstaichi's compiled 3x3 SVD, whose source is absent.  It
is replaced by LAPACK's SVD in the convention ti.svd documents (U and V proper rotations,
singular values in decreasing order, a reflection carried by the sign of the last one).
Material, stress, boundary and SVD-adjoint outputs are invariant under the remaining
freedom (simultaneous sign changes of matching U and V columns) wherever the singular
values are distinct.
"""

from __future__ import annotations

import functools
import importlib.util
import itertools
import os
import sys
import types as _pytypes

import numpy as np


# ----------------------------------------------------------------------------- values
class TiArr(np.ndarray):
    """A Taichi vector/matrix value.  ``_wb`` (array, index) makes a copy read out of a field
    write itself back on item assignment, as ``field[i].member[d] = x`` does in Taichi."""

    def __array_finalize__(self, obj):
        self._wb = None

    def _write_back(self):
        wb = self._wb
        if wb is not None:
            arr, idx = wb
            arr[idx] = np.asarray(self)

    def __setitem__(self, key, value):
        super().__setitem__(key, value)
        self._write_back()

    def fill(self, value):
        super().fill(value)
        self._write_back()

    def norm(self, eps=0):
        a = np.asarray(self)
        return np.sqrt(np.sum(a * a) + eps)

    def norm_sqr(self):
        a = np.asarray(self)
        return np.sum(a * a)

    def dot(self, other):
        return np.sum(np.asarray(self) * np.asarray(other))

    def cross(self, other):
        return np.cross(np.asarray(self), np.asarray(other)).view(TiArr)

    def outer_product(self, other):
        return np.multiply.outer(np.asarray(self), np.asarray(other)).view(TiArr)

    def determinant(self):
        a = np.asarray(self)
        if a.shape == (2, 2):
            return a[0, 0] * a[1, 1] - a[0, 1] * a[1, 0]
        assert a.shape == (3, 3)
        return (a[0, 0] * (a[1, 1] * a[2, 2] - a[2, 1] * a[1, 2])
                - a[1, 0] * (a[0, 1] * a[2, 2] - a[2, 1] * a[0, 2])
                + a[2, 0] * (a[0, 1] * a[1, 2] - a[1, 1] * a[0, 2]))

    def cast(self, dtype):
        return np.asarray(self).astype(_np_dtype(dtype)).view(TiArr)

    def max(self, *a, **k):
        return np.asarray(self).max(*a, **k)


def _val(x):
    """A fresh value (pass-by-value copy) of x."""
    if isinstance(x, np.ndarray):
        return np.array(x).view(TiArr)
    return x


# ----------------------------------------------------------------------------- dtypes
f32, f64, i32, i64, u1, u8 = np.float32, np.float64, np.int32, np.int64, np.bool_, np.uint8
f16 = np.float16


def _np_dtype(dt):
    if isinstance(dt, _VecT):
        return dt.dtype
    return np.dtype(dt).type


class _VecT:
    def __init__(self, shape, dtype):
        self.shape = tuple(shape)
        self.dtype = _np_dtype(dtype)

    def __call__(self, *a):
        return np.array(a[0] if len(a) == 1 else a, dtype=self.dtype).view(TiArr)


class _StructT:
    def __init__(self, members):
        self.members = {}
        for k, t in members.items():
            if isinstance(t, _VecT):
                self.members[k] = (t.shape, t.dtype)
            else:
                self.members[k] = ((), _np_dtype(t))

    def field(self, shape, needs_grad=False, layout=None):
        return StructField(self.members, shape, needs_grad)


class types:  # noqa: N801  (ti.types namespace)
    @staticmethod
    def vector(n, dtype):
        return _VecT((n,), dtype)

    @staticmethod
    def matrix(n, m, dtype):
        return _VecT((n, m), dtype)

    @staticmethod
    def struct(**members):
        return _StructT(members)

    @staticmethod
    def ndarray(*a, **k):
        return None


class Layout:
    SOA = "soa"
    AOS = "aos"


def template(*a, **k):
    return None


# ----------------------------------------------------------------------------- fields
def _flat_index(key):
    if key is None:  # field[None]: the element of a 0-d field
        return ()
    if not isinstance(key, tuple):
        key = (key,)
    out = []
    for k in key:
        if isinstance(k, (tuple, list, np.ndarray)):
            out.extend(int(v) for v in np.asarray(k).ravel())
        else:
            out.append(int(k))
    return tuple(out)


class _Elem:
    __slots__ = ("_f", "_i")

    def __init__(self, f, i):
        object.__setattr__(self, "_f", f)
        object.__setattr__(self, "_i", i)

    def __getattr__(self, name):
        arr = self._f._data[name]
        v = arr[self._i]
        if np.ndim(v) == 0:
            return v
        out = np.array(v).view(TiArr)
        out._wb = (arr, self._i)
        return out

    def __setattr__(self, name, value):
        self._f._data[name][self._i] = np.asarray(value)


class StructField:
    def __init__(self, members, shape, needs_grad=False):
        shape = (shape,) if np.isscalar(shape) else shape
        self.shape = tuple(int(s) for s in shape)
        self._data = {k: np.zeros(self.shape + ms, dtype=dt) for k, (ms, dt) in members.items()}
        self.grad = StructField(members, shape) if needs_grad else None

    def __getitem__(self, key):
        return _Elem(self, _flat_index(key))

    def member(self, name):
        return self._data[name]

    def fill(self, v):
        for a in self._data.values():
            a.fill(v)


class Field:
    """ti.field / ti.Vector.field of one value type."""

    def __init__(self, dtype, shape):
        if isinstance(dtype, _VecT):
            self._eshape, dt = dtype.shape, dtype.dtype
        else:
            self._eshape, dt = (), _np_dtype(dtype)
        shape = (shape,) if np.isscalar(shape) else tuple(shape)
        self.shape = tuple(int(s) for s in shape)
        self._a = np.zeros(self.shape + self._eshape, dtype=dt)

    def __getitem__(self, key):
        i = _flat_index(key)
        v = self._a[i]
        if np.ndim(v) == 0:
            return v
        out = np.array(v).view(TiArr)
        out._wb = (self._a, i)
        return out

    def __setitem__(self, key, value):
        self._a[_flat_index(key)] = np.asarray(value)

    def from_numpy(self, a):
        self._a[...] = np.asarray(a).reshape(self._a.shape)

    def to_numpy(self):
        return self._a.copy()

    def fill(self, v):
        self._a.fill(v)


def field(dtype, shape, needs_grad=False, **k):
    return Field(dtype, shape)


# ----------------------------------------------------------------------------- constructors
class Matrix:
    def __new__(cls, data, dt=None):
        return np.array(data, dtype=np.float64 if dt is None else _np_dtype(dt)).view(TiArr)

    @staticmethod
    def zero(dt, n, m=None):
        return np.zeros((n, m) if m is not None else (n,), dtype=_np_dtype(dt)).view(TiArr)

    @staticmethod
    def identity(dt, n):
        return np.eye(n, dtype=_np_dtype(dt)).view(TiArr)

    @staticmethod
    def field(n, m, dtype, shape, **k):
        return Field(_VecT((n, m), dtype), shape)


class Vector:
    def __new__(cls, data, dt=None):
        a = np.asarray(data)
        if dt is not None:
            dtype = _np_dtype(dt)
        else:
            dtype = np.int64 if a.dtype.kind in "iub" else np.float64
        return np.array(a, dtype=dtype).view(TiArr)

    @staticmethod
    def zero(dt, n):
        return np.zeros((n,), dtype=_np_dtype(dt)).view(TiArr)

    @staticmethod
    def field(n, dtype, shape, **k):
        return Field(_VecT((n,), dtype), shape)


# ----------------------------------------------------------------------------- decorators
def data_oriented(cls):
    return cls


def func(fn):
    @functools.wraps(fn)
    def call(*a, **k):
        return fn(*[_val(x) for x in a], **{n: _val(x) for n, x in k.items()})

    return call


def kernel(fn):
    ann = dict(getattr(fn, "__annotations__", {}))
    names = fn.__code__.co_varnames[: fn.__code__.co_argcount]

    def conv(name, x):
        t = ann.get(name)
        if t is f32:
            return float(np.float32(x))
        if t is f64:
            return float(x)
        if t is i32 or t is i64:
            return int(x)
        return x

    @functools.wraps(fn)
    def call(*a, **k):
        a = [conv(n, x) for n, x in zip(names, a)] + list(a[len(names):])
        k = {n: conv(n, x) for n, x in k.items()}
        return fn(*a, **k)

    call.grad = None
    return call


def static(x, *a):
    return x


# ----------------------------------------------------------------------------- loops
def ndrange(*dims):
    rs = []
    for d in dims:
        if isinstance(d, (tuple, list)):
            rs.append(range(int(d[0]), int(d[1])))
        else:
            rs.append(range(int(d)))
    return itertools.product(*rs)


def grouped(it):
    for idx in it:
        yield np.array(idx if isinstance(idx, tuple) else (idx,), dtype=np.int64).view(TiArr)


# ----------------------------------------------------------------------------- math
def _wrap(x):
    return x.view(TiArr) if isinstance(x, np.ndarray) and x.ndim else x


def max(a, b):  # noqa: A001
    return _wrap(np.maximum(a, b))


def min(a, b):  # noqa: A001
    return _wrap(np.minimum(a, b))


def abs(x):  # noqa: A001
    return _wrap(np.abs(x))


def exp(x):
    return _wrap(np.exp(x))


def log(x):
    return _wrap(np.log(x))


def sqrt(x):
    return _wrap(np.sqrt(x))


def pow(x, y):  # noqa: A001
    return _wrap(np.power(x, y))


def floor(x, dt=None):
    r = np.floor(x)
    return _wrap(r.astype(_np_dtype(dt)) if dt is not None else r)


def cast(x, dt):
    if isinstance(x, np.ndarray):
        return np.asarray(x).astype(_np_dtype(dt)).view(TiArr)
    return _np_dtype(dt)(x)


def select(c, a, b):
    return _wrap(np.where(c, a, b))


class math:  # noqa: N801
    isnan = staticmethod(np.isnan)
    isinf = staticmethod(np.isinf)


def svd(A, dt=None):
    """3x3 SVD in ti.svd's convention: A = U diag(s) V^T with U, V proper rotations,
    s in decreasing order of magnitude, the last entry carrying a reflection's sign."""
    a = np.asarray(A, dtype=np.float64)
    U, s, Vh = np.linalg.svd(a)
    V = Vh.T.copy()
    U = U.copy()
    if np.linalg.det(U) < 0:
        U[:, 2] *= -1
        s[2] *= -1
    if np.linalg.det(V) < 0:
        V[:, 2] *= -1
        s[2] *= -1
    return U.view(TiArr), np.diag(s).view(TiArr), V.view(TiArr)


# ----------------------------------------------------------------------------- genesis stubs
def _module(name, **attrs):
    m = _pytypes.ModuleType(name)
    m.__path__ = []  # every stub may act as a package
    m.__dict__.update(attrs)
    sys.modules[name] = m
    return m


class _Logger:
    def __getattr__(self, name):
        return lambda *a, **k: None


class _UID:
    _n = 0

    def __init__(self):
        _UID._n += 1
        self.v = _UID._n


class GenesisException(Exception):
    pass


def _raise_exception(msg="", *a):
    raise GenesisException(msg)


class RBC:
    pass


class _Anything:
    """Annotation placeholder (array_class.GeomsState and friends)."""


def install(precision: str = "64"):
    """Register this module as ``gstaichi`` and stub modules for the rest of ``genesis``."""
    ti = sys.modules[__name__]
    sys.modules["gstaichi"] = ti
    tf = f64 if precision == "64" else f32
    eps = float(np.maximum(1e-15, np.finfo(tf).eps))  # EPS = max(eps, finfo(np_float).eps)
    gs = _module(
        "genesis",
        ti_float=tf, np_float=tf, ti_int=i32, np_int=np.int32, ti_bool=u1, np_bool=np.bool_,
        ti_vec2=types.vector(2, tf), ti_vec3=types.vector(3, tf), ti_vec4=types.vector(4, tf),
        ti_mat3=types.matrix(3, 3, tf), ti_mat4=types.matrix(4, 4, tf), ti_ivec3=types.vector(3, i32),
        EPS=eps, platform="Linux", logger=_Logger(), raise_exception=_raise_exception, UID=_UID, List=list,
        assert_built=lambda fn: fn, device="cpu", GenesisException=GenesisException,
    )
    try:
        import torch

        gs.tc_float = torch.float64 if precision == "64" else torch.float32
        gs.tc_int = torch.int32
        gs.tc_bool = torch.bool
    except ImportError:
        pass
    _module("genesis.repr_base", RBC=RBC)
    _module("genesis.utils")
    _module("genesis.utils.misc", DeprecationError=DeprecationWarning, ti_to_torch=None, tensor_to_array=None)
    _module("genesis.utils.repr", brief=repr)
    _module("genesis.utils.geom", ti_inv_transform_by_trans_quat=None, ti_transform_by_trans_quat=None)
    _module("genesis.utils.sdf_decomp")
    arr = _module("genesis.utils.array_class", V=field)
    for n in ("GeomsState", "GeomsInfo", "LinksState", "RigidGlobalInfo", "SDFInfo"):
        setattr(arr, n, _Anything)
    _module("genesis.options")
    _module("genesis.options.solvers", MPMOptions=object, LegacyCouplerOptions=object)
    _module("genesis.engine")
    _module("genesis.engine.entities", MPMEntity=object)
    _module("genesis.engine.entities.base_entity", Entity=object)
    _module("genesis.engine.states")
    _module("genesis.engine.states.solvers", MPMSolverState=object)
    for pkg in ("genesis.engine.boundaries", "genesis.engine.solvers", "genesis.engine.couplers",
                "genesis.engine.materials", "genesis.engine.materials.MPM"):
        _module(pkg)
    gs.utils = sys.modules["genesis.utils"]
    return gs


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


class Reference:
    """The reference's MPM classes, imported unchanged from a Genesis checkout at `root`."""

    def __init__(self, root: str, precision: str = "64"):
        self.root = root
        self.gs = install(precision)
        g = os.path.join(root, "genesis", "engine")
        bnd = _load("genesis.engine.boundaries.boundaries", os.path.join(g, "boundaries", "boundaries.py"))
        sys.modules["genesis.engine.boundaries"].CubeBoundary = bnd.CubeBoundary
        _load("genesis.engine.materials.base", os.path.join(g, "materials", "base.py"))
        mats = {}
        for n in ("base", "elastic", "elasto_plastic", "liquid", "sand", "snow", "muscle"):
            mats[n] = _load(f"genesis.engine.materials.MPM.{n}", os.path.join(g, "materials", "MPM", f"{n}.py"))
        self.Elastic = mats["elastic"].Elastic
        self.ElastoPlastic = mats["elasto_plastic"].ElastoPlastic
        self.Liquid = mats["liquid"].Liquid
        self.Sand = mats["sand"].Sand
        self.Snow = mats["snow"].Snow
        self.Muscle = mats["muscle"].Muscle
        _load("genesis.engine.solvers.base_solver", os.path.join(g, "solvers", "base_solver.py"))
        self.mpm_solver = _load("genesis.engine.solvers.mpm_solver", os.path.join(g, "solvers", "mpm_solver.py"))
        self.coupler = _load("genesis.engine.couplers.legacy_coupler",
                             os.path.join(g, "couplers", "legacy_coupler.py"))
        self.CubeBoundary = bnd.CubeBoundary
        self.backward_svd = self.mpm_solver.backward_svd


class _NS:
    def __init__(self, **k):
        self.__dict__.update(k)


class _Entity:
    """What MPMEntity._add_to_solver does for a particle block (mpm_entity.py): one
    _kernel_add_particles call with the material's index, default Jp and density."""

    def __init__(self, material, pos, active=True):
        self.material = material
        self.pos = np.asarray(pos, dtype=np.float64)
        self.n_particles = self.pos.shape[0]
        self.n_vverts = 0
        self.n_vfaces = 0
        self.active = active
        self.particle_start = 0

    def _add_to_solver(self, solver):
        solver._kernel_add_particles(0, self.active, self.particle_start, self.n_particles, self.material._idx,
                                     self.material._default_Jp, self.material._rho, self.pos)


class Scene:
    """One MPM scene driven through the reference's own MPMSolver and LegacyCoupler code:
    MPMSolver.__init__ (derived constants, boundary), add_material, build's field set-up and
    _kernel_add_particles, then per substep exactly Simulator.substep's order
    (coupler.preprocess, reset_grid_and_grad + compute_F_tmp + svd + p2g, mpm_grid_op, g2p +
    the NaN check) followed by the frame copy of save_ckpt."""

    def __init__(self, ref: Reference, grid_density, lower_bound, upper_bound, particle_size, dt, gravity,
                 blocks):
        self.ref = ref
        opts = _NS(dt=dt, gravity=tuple(gravity), grid_density=grid_density, particle_size=particle_size,
                   upper_bound=tuple(upper_bound), lower_bound=tuple(lower_bound), enable_CPIC=False)
        scene = _NS(vis_options=_NS(n_support_neighbors=4), _is_built=False)
        sim = _NS(substeps=1, substeps_local=1, _B=1, requires_grad=False, cur_t=0.0)
        S = ref.mpm_solver.MPMSolver
        s = S.__new__(S)
        S.__init__(s, scene, sim, opts)
        ents = []
        start = 0
        for mat, pos in blocks:
            s.add_material(mat)
            e = _Entity(mat, pos)
            e.particle_start = start
            start += e.n_particles
            ents.append(e)
        s._entities = ents
        # MPMSolver.build (mpm_solver.py:172-209) without the entity classes
        s._B = 1
        s._n_particles = start
        s._n_vverts = 0
        s._n_vfaces = 0
        scene._is_built = True
        s.init_particle_fields()
        s.init_grid_fields()
        s.init_vvert_fields()
        s.init_ckpt()
        for e in ents:
            e._add_to_solver(s)
        grav = np.tile(np.asarray(gravity, dtype=np.float64), (1, 1))
        s._gravity = field(self.ref.gs.ti_vec3, (1,))
        s._gravity.from_numpy(grav)
        rigid = _NS(is_active=False, n_geoms=0, geoms_state=None, geoms_info=None, links_state=None,
                    _rigid_global_info=None, sdf=_NS(_sdf_info=None), collider=_NS(_collider_static_config=None))
        off = dict(is_active=False)
        sim2 = _NS(mpm_solver=s, rigid_solver=rigid, tool_solver=_NS(**off), avatar_solver=_NS(**off),
                   sph_solver=_NS(**off), pbd_solver=_NS(**off), fem_solver=_NS(**off), sf_solver=_NS(**off),
                   cur_t=0.0)
        C = ref.coupler.LegacyCoupler
        cp = C.__new__(C)
        C.__init__(cp, sim2, _NS())
        cp._rigid_mpm = cp._rigid_sph = cp._rigid_pbd = cp._rigid_fem = False
        cp._mpm_sph = cp._mpm_pbd = cp._fem_mpm = cp._fem_sph = False
        s._coupler = cp
        s._sim.rigid_solver = rigid
        s._sim.coupler = _NS(rigid_solver=rigid)
        self.solver, self.coupler, self.rigid = s, cp, rigid

    # state access (frame 0) ------------------------------------------------------------
    def state(self, f=0):
        p = self.solver.particles
        out = {k: p.member(k)[f, :, 0].copy() for k in ("pos", "vel", "C", "F", "Jp")}
        out["active"] = self.solver.particles_ng.member("active")[f, :, 0].copy()
        return out

    def set_state(self, **kw):
        p = self.solver.particles
        for k, v in kw.items():
            if k == "active":
                self.solver.particles_ng.member("active")[0, :, 0] = v
            else:
                p.member(k)[0, :, 0] = v

    def grid(self, f=0):
        g = self.solver.grid
        return g.member("mass")[f, :, :, :, 0].copy(), g.member("vel_in")[f, :, :, :, 0].copy()

    def substep(self):
        s, cp, r = self.solver, self.coupler, self.rigid
        f = 0
        # Simulator.substep (simulator.py:313-317)
        cp.preprocess(f)
        s.substep_pre_coupling(f)
        grid = self.grid(f)
        cp.couple(f)
        s.substep_post_coupling(f)
        # Simulator.step -> save_ckpt -> copy_frame(substeps_local, 0) (mpm_solver.py:663-664)
        s.copy_frame(1, 0)
        return grid
