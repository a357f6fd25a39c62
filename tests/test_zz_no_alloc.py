"""GPU test of the allocation-free sort entry point (mpm_radix_sort_pairs_noalloc).

That entry point exists for callers that cannot allocate device memory —
code inside a stream-ordered pipeline that must not stall on cudaMalloc or
cudaFree, hosts that reserve the device budget up front, hot paths held to an
allocation-free guarantee.  It keeps its scratch in a fixed device array of
the library (limit 1,048,576 pairs).  Here it is called through the C ABI
twice in a row on device buffers and its output is compared, bit for bit
(integer sort), with the allocating entry point mpm_radix_sort_pairs_device
on the same inputs; oversized requests must be rejected without touching
the buffers.  This file is collected last so that a run stopping at the
first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 1 << 20


def _lib():
    from molla_b200 import _ffi
    return _ffi.lib()


def _sort_reference(engine, keys, vals, bits):
    import torch
    k = torch.from_numpy(keys.astype(np.int32)).cuda()
    v = torch.from_numpy(vals.astype(np.int32)).cuda()
    torch.cuda.synchronize()
    rc = _lib().mpm_radix_sort_pairs_device(engine._h, ctypes.c_void_p(k.data_ptr()), ctypes.c_void_p(v.data_ptr()),
                                            keys.shape[0], bits, None)
    assert rc == 0
    _lib().mpm_engine_synchronize(engine._h)
    return k.cpu().numpy().view(np.uint32), v.cpu().numpy().view(np.uint32)


def _sort_noalloc(keys, vals, bits):
    import torch
    k = torch.from_numpy(keys.astype(np.int32)).cuda()
    v = torch.from_numpy(vals.astype(np.int32)).cuda()
    torch.cuda.synchronize()
    rc = _lib().mpm_radix_sort_pairs_noalloc(ctypes.c_void_p(k.data_ptr()), ctypes.c_void_p(v.data_ptr()),
                                             keys.shape[0], bits, None)
    assert rc == 0
    torch.cuda.synchronize()
    return k.cpu().numpy().view(np.uint32), v.cpu().numpy().view(np.uint32)


def test_noalloc_sort_matches_allocating_sort_twice(engine):
    rng = np.random.default_rng(2024)
    cases = [(LIMIT, 32), (300_001, 18)]  # two calls in a row, different sizes and widths
    for n, bits in cases:
        keys = rng.integers(0, 1 << bits, size=n, dtype=np.uint64).astype(np.uint32)
        vals = rng.permutation(n).astype(np.uint32)
        got_k, got_v = _sort_noalloc(keys, vals, bits)
        ref_k, ref_v = _sort_reference(engine, keys, vals, bits)
        assert np.array_equal(got_k, ref_k)
        assert np.array_equal(got_v, ref_v)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(got_k, keys[order]) and np.array_equal(got_v, vals[order])


def test_noalloc_sort_rejects_oversized_input():
    import torch
    from molla_b200 import _ffi
    k = torch.arange(LIMIT + 1, dtype=torch.int32, device="cuda").flip(0)
    v = torch.arange(LIMIT + 1, dtype=torch.int32, device="cuda")
    before = k.clone()
    rc = _lib().mpm_radix_sort_pairs_noalloc(ctypes.c_void_p(k.data_ptr()), ctypes.c_void_p(v.data_ptr()),
                                             LIMIT + 1, 32, None)
    torch.cuda.synchronize()
    assert rc == _ffi.MPM_ERR_INVALID
    assert "exceeds" in _ffi.last_error()
    assert torch.equal(k, before)
