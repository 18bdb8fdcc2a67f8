"""bh_radix_sort_pairs_noalloc: the radix sort for callers that cannot
allocate device memory where they sort (code that must not stall the device
with cudaFree, or a plugin whose host framework owns the device memory).  Its
scratch is a static array inside the library, so its results must equal those
of the sorter-based entry point (bh_radix_sort_pairs) bit for bit, call after
call, even though every call reuses the array the previous call left dirty;
and a call must not change the device's free memory.

This file is collected last on purpose: a failure here leaves every other
test already run."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import to_device

pytestmark = pytest.mark.gpu

MAX_PAIRS = 262144  # BH_NOALLOC_SORT_MAX in include/sorting.h
TIMEOUT = 8         # BH_ERR_TIMEOUT


def _keys(n, seed, key_bits=64):
    """Keys with key_bits significant bits (the sort's contract: the bits
    above key_bits are zero), duplicates included."""
    rng = np.random.default_rng(seed)
    keys = (rng.integers(0, 1 << 12, n, dtype=np.uint64) << np.uint64(44)) | rng.integers(0, 1 << 30, n,
                                                                                         dtype=np.uint64)
    if key_bits < 64:
        keys &= np.uint64((1 << key_bits) - 1)
    keys[::9] = keys[3]  # duplicates: stability matters
    return keys, rng.permutation(n).astype(np.uint32)


def _noalloc(engine, torch, kin, vin, key_bits):
    kout, vout = torch.empty_like(kin), torch.empty_like(vin)
    torch.cuda.synchronize()
    rc = engine.lib().bh_radix_sort_pairs_noalloc(kin.data_ptr(), kout.data_ptr(), vin.data_ptr(), vout.data_ptr(),
                                                  kin.shape[0], key_bits, None)
    torch.cuda.synchronize()
    return rc, kout, vout


@pytest.mark.parametrize("n", [100_000, MAX_PAIRS])
@pytest.mark.parametrize("key_bits", [64, 30, 20, 8])  # 8, 4, 3 and 1 digit passes
def test_noalloc_sort_matches_sorter_twice(torch_cuda, engine, n, key_bits):
    """Two calls in a row against the sorter-based sort.  Odd pass counts
    leave an intermediate result in the static array's key/value buffers; the
    second call runs on what the first left behind and must not change the
    device's free memory."""
    torch = torch_cuda
    for call in range(2):
        keys, vals = _keys(n, 1000 * n + 10 * key_bits + call, key_bits)
        kin, vin = to_device(torch, keys.view(np.int64)), to_device(torch, vals.view(np.int32))
        free0 = torch.cuda.mem_get_info()[0]
        rc, kout, vout = _noalloc(engine, torch, kin, vin, key_bits)  # the first call works in a fresh process
        free1 = torch.cuda.mem_get_info()[0]
        assert rc == 0, engine.status_string(rc)
        assert engine.lib().bh_radix_sort_noalloc_errors(None, None) == 0
        if call == 1:
            assert free1 == free0  # allocates nothing
        kref, vref = torch.empty_like(kin), torch.empty_like(vin)
        engine.radix_sort_pairs(kin, vin, kref, vref, key_bits=key_bits)
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
    assert engine.lib().bh_last_error() == 1


def test_noalloc_sort_reports_device_timeout(torch_cuda, engine):
    """Failure detection without a fault: a look-back wait on the static
    array's status words whose predecessor never publishes gives up; the
    error query reports BH_ERR_TIMEOUT, and the next sort clears it."""
    torch = torch_cuda
    assert engine.lib().bh_selftest_noalloc_timeout(None) == 0
    bits = np.zeros(1, np.int32)
    assert engine.lib().bh_radix_sort_noalloc_errors(bits.ctypes.data, None) == TIMEOUT
    assert bits[0] == 1 << (TIMEOUT - 1)
    keys, vals = _keys(5000, 3)
    kin, vin = to_device(torch, keys.view(np.int64)), to_device(torch, vals.view(np.int32))
    rc, kout, vout = _noalloc(engine, torch, kin, vin, 64)
    assert rc == 0 and engine.lib().bh_radix_sort_noalloc_errors(None, None) == 0
    assert np.array_equal(vout.cpu().numpy().view(np.uint32), vals[np.argsort(keys, kind="stable")])
