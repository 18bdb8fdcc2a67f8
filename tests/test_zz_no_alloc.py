"""bh_radix_sort_pairs_noalloc: the radix sort for callers that cannot
allocate device memory where they sort (code that must not stall the device
with cudaFree, or a plugin whose host framework owns the device memory).  Its scratch is a static array inside
the library, so its results must equal those of the sorter-based entry point
(bh_radix_sort_pairs) bit for bit, call after call, even though every call
reuses the array the previous call left dirty.

This file is collected last on purpose: a failure here leaves every other
test already run."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import to_device

pytestmark = pytest.mark.gpu

MAX_PAIRS = 262144  # BH_NOALLOC_SORT_MAX in include/sorting.h


def _keys(n, seed):
    rng = np.random.default_rng(seed)
    keys = (rng.integers(0, 1 << 12, n, dtype=np.uint64) << np.uint64(44)) | rng.integers(0, 1 << 30, n,
                                                                                         dtype=np.uint64)
    keys[::9] = keys[3]  # duplicates: stability matters
    return keys, rng.permutation(n).astype(np.uint32)


def _noalloc(engine, torch, kin, vin, key_bits):
    kout, vout = torch.empty_like(kin), torch.empty_like(vin)
    rc = engine.lib().bh_radix_sort_pairs_noalloc(kin.data_ptr(), kout.data_ptr(), vin.data_ptr(), vout.data_ptr(),
                                                  kin.shape[0], key_bits, None)
    torch.cuda.synchronize()
    return rc, kout, vout


@pytest.mark.parametrize("n", [100_000, MAX_PAIRS])
def test_noalloc_sort_matches_sorter_twice(torch_cuda, engine, n):
    torch = torch_cuda
    for call in range(2):  # the second call runs on the scratch the first left behind
        keys, vals = _keys(n, 1000 * n + call)
        kin, vin = to_device(torch, keys.view(np.int64)), to_device(torch, vals.view(np.int32))
        rc, kout, vout = _noalloc(engine, torch, kin, vin, 64)  # first: works in a fresh process
        assert rc == 0, engine.status_string(rc)
        kref, vref = torch.empty_like(kin), torch.empty_like(vin)
        engine.radix_sort_pairs(kin, vin, kref, vref, key_bits=64)
        assert torch.equal(kout, kref) and torch.equal(vout, vref)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(vout.cpu().numpy().view(np.uint32), vals[order])
        assert np.array_equal(kin.cpu().numpy().view(np.uint64), keys)  # inputs untouched


def test_noalloc_sort_rejects_oversize(torch_cuda, engine):
    torch = torch_cuda
    keys, vals = _keys(MAX_PAIRS + 1, 7)
    kin, vin = to_device(torch, keys.view(np.int64)), to_device(torch, vals.view(np.int32))
    rc, _, _ = _noalloc(engine, torch, kin, vin, 64)
    assert rc == 1  # BH_ERR_INVALID: beyond the static scratch
