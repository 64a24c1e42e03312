"""Process-wide settings made by gs.init (genesis/__init__.py:54-330)."""

import numpy as np
import torch

initialized = False
backend = None
precision = "32"
seed = None
debug = False
EPS = float(np.finfo(np.float32).eps)
device = None
tc_float = torch.float32
np_float = np.float32
rng = np.random.default_rng()
