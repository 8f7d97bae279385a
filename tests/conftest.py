"""Shared fixtures. `-m gpu` tests need a B200; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

SIGNED = {1: np.int8, 2: np.int16, 4: np.int32, 8: np.int64}
UNSIGNED = {1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device (B200)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle

    return Oracle.instance()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference

    if not Reference.available():
        pytest.skip("reference CPU build (oracle/_ref) not present")
    return Reference()


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def to_dev(a: np.ndarray):
    """numpy (any unsigned width) -> CUDA tensor holding the same bytes."""
    import torch

    a = np.ascontiguousarray(a)
    signed = SIGNED[a.dtype.itemsize]
    return torch.from_numpy(a.view(signed).copy()).to("cuda")


def from_dev(t, elem_bytes: int) -> np.ndarray:
    return t.cpu().numpy().view(UNSIGNED[elem_bytes])


def dev_empty(n: int, elem_bytes: int, fill: int | None = None):
    import torch

    dt = {1: torch.int8, 2: torch.int16, 4: torch.int32, 8: torch.int64}[elem_bytes]
    t = torch.empty(max(n, 1), dtype=dt, device="cuda")
    if fill is not None:
        t.view(torch.uint8).fill_(fill)
    return t
