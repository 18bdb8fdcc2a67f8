"""Shared fixtures.  Tests marked `gpu` need a CUDA device (a B200); the rest
run on the CPU.  The oracle (oracle/) is the checker, never the thing
checked."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); parity tests proper")


@pytest.fixture(scope="session")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.init()
    return torch


@pytest.fixture(scope="session")
def engine():
    import cudagravitydemo_b200 as bh
    bh.lib()
    return bh


@pytest.fixture(scope="session")
def oracle():
    from oracle import build, cpu
    build.build_oracle()
    return cpu


class _DevView:
    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def dev_to_host(ptr: int, shape, dtype) -> np.ndarray:
    """Copy device memory at `ptr` into a new numpy array."""
    import torch
    dtype = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dtype.itemsize
    t = torch.as_tensor(_DevView(ptr, (nbytes,), "|u1"), device="cuda")
    torch.cuda.synchronize()
    return t.cpu().numpy().view(dtype).reshape(shape).copy()


def to_device(torch, arr: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(arr)).cuda()


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def node_fields_equal(a: np.ndarray, b: np.ndarray, skip_root_parent: bool = True) -> list[str]:
    """Names of node fields that differ (massData compared bit for bit)."""
    bad = []
    if a.shape != b.shape:
        return [f"count {a.shape} vs {b.shape}"]
    for f in ("path", "first", "count", "child", "level"):
        if not np.array_equal(a[f], b[f]):
            bad.append(f)
    pa, pb = a["parent"].copy(), b["parent"].copy()
    if skip_root_parent and len(pa):
        pa[0] = pb[0] = -1
    if not np.array_equal(pa, pb):
        bad.append("parent")
    if not np.array_equal(a["mass"].view(np.uint32), b["mass"].view(np.uint32)):
        bad.append("mass")
    return bad
