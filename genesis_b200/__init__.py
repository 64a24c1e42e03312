"""genesis_b200: a B200-native (sm_100a) MLS-MPM substep behind Genesis's MPM API.

    import genesis_b200 as gs
    gs.init(backend=gs.gpu, precision="32")
    scene = gs.Scene(sim_options=gs.options.SimOptions(dt=1e-4, substeps=10),
                     mpm_options=gs.options.MPMOptions(lower_bound=(0, 0, 0), upper_bound=(1, 1, 1)))
    cube = scene.add_entity(gs.morphs.Box(lower=(0.4,) * 3, upper=(0.6,) * 3),
                            material=gs.materials.MPM.Elastic(E=1e5, nu=0.3))
    scene.build()
    scene.step()
"""

from __future__ import annotations

import logging

import numpy as np
import torch

from . import _globals
from . import force_fields, materials, morphs, options, surfaces, textures
from .engine.emitter import Emitter
from .engine.scene import Scene
from .exceptions import GenesisException
from .creation_ops import *  # noqa: F401,F403  gs.tensor, gs.zeros, ... (genesis/grad/creation_ops.py)
from .creation_ops import from_torch

__version__ = "0.1.0"

gpu = "gpu"
cuda = "cuda"
cpu = "cpu"

tc_float = torch.float32
np_float = np.float32
tc_int = torch.int32
np_int = np.int32
tc_bool = torch.bool
ACTIVE = 1
INACTIVE = 0


def init(seed=None, precision="32", debug=False, eps=1e-15, backend=None, logging_level=None, **_ignored):
    """gs.init (genesis/__init__.py:54-330) for the CUDA path: float32 only, GPU only."""
    global EPS, device
    if backend is None:
        backend = gpu
    if backend == cpu:
        raise GenesisException(
            "genesis_b200 has no CPU backend: the MPM path runs only as sm_100a CUDA kernels (no CPU fallback)."
        )
    if backend not in (gpu, cuda):
        raise GenesisException(f"Unsupported backend: {backend}")
    if str(precision) != "32":
        raise GenesisException("genesis_b200 computes in float32 only (precision='32').")
    if logging_level is not None:
        logging.getLogger("genesis_b200").setLevel(logging_level.upper() if isinstance(logging_level, str) else logging_level)
    _globals.precision = "32"
    _globals.backend = backend
    _globals.debug = debug
    _globals.seed = seed
    # EPS = max(eps, finfo(float32).eps) (genesis/__init__.py:205-206)
    _globals.EPS = max(float(eps), float(np.finfo(np.float32).eps))
    _globals.rng = np.random.default_rng(seed)
    if seed is not None:
        torch.manual_seed(seed)
    _globals.device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cuda")
    _globals.initialized = True
    EPS = _globals.EPS
    device = _globals.device


def destroy():
    _globals.initialized = False


EPS = _globals.EPS
device = None

__all__ = ["init", "destroy", "Scene", "Emitter", "GenesisException", "materials", "morphs", "options", "surfaces", "textures", "gpu", "cpu", "cuda"]
