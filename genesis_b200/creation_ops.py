"""gs.tensor, gs.zeros, ... (genesis/grad/creation_ops.py): torch's creation functions with the
reference's conventions -- the tensor lands on the device gs.init chose, float dtypes become
float32 and integer dtypes int32, the result is a new leaf (detached from its source) that
requires grad when asked.  Here they are plain torch tensors: a differentiable scene's
gradients flow through torch autograd nodes, so no scene-aware tensor type is needed."""

from __future__ import annotations

import functools
import sys

import torch

from . import _globals
from .exceptions import GenesisException

_OPS = (torch.tensor, torch.asarray, torch.as_tensor, torch.as_strided, torch.from_numpy, torch.zeros,
        torch.zeros_like, torch.ones, torch.ones_like, torch.arange, torch.linspace, torch.logspace, torch.eye,
        torch.empty, torch.empty_like, torch.empty_strided, torch.full, torch.full_like, torch.rand,
        torch.rand_like, torch.randn, torch.randn_like, torch.randint, torch.randint_like, torch.randperm)


def from_torch(torch_tensor, dtype=None, requires_grad=False, detach=True, scene=None):
    """A copy of torch_tensor on the device in float32 / int32 / bool; with detach=True (the
    default) a new leaf not connected to torch_tensor's graph."""
    if dtype is None:
        dtype = torch_tensor.dtype
    if dtype in (float, torch.float16, torch.bfloat16, torch.float32, torch.float64):
        dtype = torch.float32
    elif dtype in (int, torch.int8, torch.int16, torch.int32, torch.int64, torch.uint8):
        dtype = torch.int32
    elif dtype in (bool, torch.bool):
        dtype = torch.bool
    else:
        raise GenesisException(f"Unsupported dtype: {dtype}")
    if torch_tensor.requires_grad and not detach and not requires_grad:
        requires_grad = True  # a tensor kept in its parent's graph stays differentiable
    t = torch_tensor.to(device=_globals.device, dtype=dtype).clone()
    if detach:
        t = t.detach()
    if requires_grad:
        t.requires_grad_()
    return t


def _wrap(op):
    @functools.wraps(op)
    def wrapper(*args, dtype=None, requires_grad=False, scene=None, **kwargs):
        if "device" in kwargs:
            raise GenesisException("Device selection not supported. All genesis tensors are on the GPU.")
        if not _globals.initialized:
            raise GenesisException("Genesis not initialized yet.")
        t = op(*args) if op is torch.from_numpy else op(*args, **kwargs)
        return from_torch(t, dtype, requires_grad, detach=True, scene=scene)

    return wrapper


for _op in _OPS:
    setattr(sys.modules[__name__], _op.__name__, _wrap(_op))

__all__ = ["from_torch"] + [op.__name__ for op in _OPS]
