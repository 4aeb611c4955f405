"""The allocation-free post-GKR entry point against the allocating one.

bitz_post_gkr_prove_noalloc serves callers that cannot allocate device memory
(a fixed memory budget owned by another allocator, a request path that must not
allocate): it runs the same sumcheck on a fixed device array inside the
library. It must give the same
point, value and transcript bytes as bitz_post_gkr_prove, on consecutive calls
that reuse the same array. This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import bitz_b200 as bz
from bitz_b200 import _lib
from oracle import ffi as of

pytestmark = pytest.mark.gpu

_u64p = ctypes.POINTER(ctypes.c_uint64)


def _claim(seed, log_rows, log_cols):
    rng = np.random.default_rng(seed)
    rows = rng.integers(0, 2**64, size=(1 << log_rows, 2), dtype=np.uint64)
    cols = rng.integers(0, 2**64, size=(1 << log_cols, 2), dtype=np.uint64)
    packed = rng.integers(0, 2**64, size=((1 << (log_rows - 7)) << log_cols, 2), dtype=np.uint64)
    return rows, cols, packed, of.weighted_sum(rows, cols, packed)


def _noalloc(rows, cols, packed, target, security, ts):
    import torch
    lib = _lib.load()
    d_rows = torch.from_numpy(rows.view(np.int64)).cuda()
    d_cols = torch.from_numpy(cols.view(np.int64)).cuda()
    d_packed = torch.from_numpy(packed.view(np.int64)).cuda()
    torch.cuda.synchronize()
    lr = rows.shape[0].bit_length() - 1
    lc = cols.shape[0].bit_length() - 1
    tgt = np.ascontiguousarray(target, dtype=np.uint64)
    point = np.zeros((lr + lc, 2), dtype=np.uint64)
    value = np.zeros(2, dtype=np.uint64)
    rc = lib.bitz_post_gkr_prove_noalloc(
        ctypes.c_void_p(d_rows.data_ptr()), lr, ctypes.c_void_p(d_cols.data_ptr()), lc,
        tgt.ctypes.data_as(_u64p), ctypes.c_void_p(d_packed.data_ptr()), security, ts.handle, None,
        point.ctypes.data_as(_u64p), value.ctypes.data_as(_u64p))
    return rc, point, value


@pytest.mark.parametrize("security", [100, 128])
def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(security):
    of.lib().o_set_clmul_mode(1)
    for seed, (lr, lc) in enumerate([(16, 2), (12, 3)]):
        rows, cols, packed, target = _claim(100 + seed, lr, lc)
        ref_ts = bz.build_prover(b"no-alloc", b"call")
        ref_point, ref_value = bz.post_gkr_prove(rows, cols, target, packed, security, ref_ts)
        ts = bz.build_prover(b"no-alloc", b"call")
        rc, point, value = _noalloc(rows, cols, packed, target, security, ts)
        assert rc == 0, _lib.load().bitz_last_error()
        assert np.array_equal(point, ref_point)
        assert np.array_equal(value, ref_value)
        assert ts.narg() == ref_ts.narg()
    of.lib().o_set_clmul_mode(0)


def test_noalloc_rejects_claims_beyond_its_scratch():
    rows, cols, packed, target = _claim(7, 14, 7)  # 2^21 bits > 2^20
    rc, _, _ = _noalloc(rows, cols, packed, target, 100, bz.build_prover(b"s", b"i"))
    assert rc == 7  # BZ_ERR_SCRATCH
    assert b"at most 20" in _lib.load().bitz_last_error()


def test_noalloc_takes_no_device_memory():
    """After a warm-up call, a second call leaves the device's free memory as
    it was: nothing is allocated on the request path."""
    import torch
    rows, cols, packed, target = _claim(11, 14, 3)
    d_rows = torch.from_numpy(rows.view(np.int64)).cuda()
    d_cols = torch.from_numpy(cols.view(np.int64)).cuda()
    d_packed = torch.from_numpy(packed.view(np.int64)).cuda()
    lib = _lib.load()
    tgt = np.ascontiguousarray(target, dtype=np.uint64)
    results = []

    def call():
        ts = bz.build_prover(b"no-alloc", b"memory")
        point = np.zeros((17, 2), dtype=np.uint64)
        value = np.zeros(2, dtype=np.uint64)
        rc = lib.bitz_post_gkr_prove_noalloc(
            ctypes.c_void_p(d_rows.data_ptr()), 14, ctypes.c_void_p(d_cols.data_ptr()), 3,
            tgt.ctypes.data_as(_u64p), ctypes.c_void_p(d_packed.data_ptr()), 100, ts.handle,
            None, point.ctypes.data_as(_u64p), value.ctypes.data_as(_u64p))
        assert rc == 0, lib.bitz_last_error()
        results.append((point.copy(), value.copy(), ts.narg()))

    torch.cuda.synchronize()
    call()  # warm-up: loads the kernels and sets up the array's address
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    free_before, _ = torch.cuda.mem_get_info()
    call()
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    assert np.array_equal(results[0][0], results[1][0])
    assert np.array_equal(results[0][1], results[1][1])
    assert results[0][2] == results[1][2]
