"""gs.tensor, gs.zeros, ... follow the reference's creation ops (genesis/grad/creation_ops.py):
float32 / int32 / bool dtypes, a new leaf, requires_grad on request, no device argument, and
nothing before gs.init.  Run here with the device globals pointed at the CPU."""

import numpy as np
import pytest
import torch

import genesis_b200 as gs
from genesis_b200 import _globals


@pytest.fixture
def on_cpu(monkeypatch):
    monkeypatch.setattr(_globals, "initialized", True)
    monkeypatch.setattr(_globals, "device", torch.device("cpu"))


def test_dtypes_leaf_and_requires_grad(on_cpu):
    t = gs.tensor([1.0, 2.0], requires_grad=True)
    assert t.dtype == torch.float32 and t.requires_grad and t.is_leaf
    assert gs.zeros(3, dtype=torch.float64).dtype == torch.float32
    assert gs.arange(4).dtype == torch.int32 and gs.ones(2, dtype=bool).dtype == torch.bool
    assert gs.from_numpy(np.arange(3.0)).dtype == torch.float32
    src = torch.ones(2, requires_grad=True)
    d = gs.from_torch(src * 2)
    assert d.is_leaf and not d.requires_grad  # detached from its source by default
    kept = gs.from_torch(src * 2, detach=False)
    assert kept.requires_grad and not kept.is_leaf
    with pytest.raises(gs.GenesisException):
        gs.zeros(3, device="cpu")


def test_refused_before_init(monkeypatch):
    monkeypatch.setattr(_globals, "initialized", False)
    with pytest.raises(gs.GenesisException):
        gs.tensor([1.0])
