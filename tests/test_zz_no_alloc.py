"""rw_tree_unique_noalloc: duplicate removal for callers that cannot allocate
GPU memory (their device memory is all handed out by their own pool, or they
run where the driver's allocation calls are off limits).  It must give exactly
what the allocating entry point rw_tree_run_stage3 gives, call after call,
although every call reuses one scratch array compiled into the library.

This file is named to be collected last, so that a run stopping at the first
failure has run every other test first.  It also passes alone."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def sorted_keys_with_runs(n, seed, key_bits):
    rng = np.random.default_rng(seed)
    top = (1 << 30) if key_bits == 32 else (1 << 63)
    distinct = rng.integers(0, top, size=max(1, n // 3), dtype=np.uint64)
    keys = rng.choice(distinct, size=n)  # about three copies of each key
    keys = np.sort(keys).astype(np.uint32 if key_bits == 32 else np.uint64)
    return keys


def via_stage3(rw, keys, key_bits):
    """The existing, allocating entry point (AppData + ImStorage)."""
    import torch
    n = keys.size
    app = rw.AppData(n, key_bits, points=np.zeros((n, 4), np.float32))
    app.u_morton_keys_alt.copy_(torch.from_numpy(keys.view(np.int32 if key_bits == 32 else np.int64)))
    im = rw.ImStorage(n, key_bits)
    rw.run_stage3(app, im)
    u = app.get_n_unique()
    return u, app.u_morton_keys[:u].cpu().numpy()


def via_noalloc(rw, keys, key_bits):
    """The no-allocation entry point, called through the C ABI."""
    import torch
    n = keys.size
    it = torch.int32 if key_bits == 32 else torch.int64
    d_in = torch.from_numpy(keys.view(np.int32 if key_bits == 32 else np.int64)).cuda()
    d_out = torch.zeros(n, dtype=it, device="cuda")
    count = ctypes.c_uint32(0)
    rc = rw.lib().rw_tree_unique_noalloc(
        ctypes.c_void_p(d_in.data_ptr()), ctypes.c_void_p(d_out.data_ptr()),
        ctypes.c_uint32(n), ctypes.c_int32(key_bits), ctypes.byref(count),
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, rw.lib().rw_tree_last_error()
    u = count.value
    return u, d_out[:u].cpu().numpy()


@pytest.mark.parametrize("key_bits", [32, 64])
def test_noalloc_unique_equals_stage3_two_calls_in_a_row(rw, key_bits):
    # a large call then a smaller one, back to back on the one scratch array
    # inside the library: each must give exactly what stage 3 gives
    for n, seed in ((1_000_003, 11), (77_777, 12)):
        keys = sorted_keys_with_runs(n, seed, key_bits)
        want_u, want = via_stage3(rw, keys, key_bits)
        got_u, got = via_noalloc(rw, keys, key_bits)
        assert got_u == want_u == np.unique(keys).size
        assert got.tobytes() == want.tobytes()


def test_noalloc_rejects_sizes_beyond_its_scratch(rw):
    limit = 1 << 26  # RW_NOALLOC_MAX_KEYS
    count = ctypes.c_uint32(0)
    dummy = ctypes.c_void_p(16)  # never dereferenced: the size check comes first
    rc = rw.lib().rw_tree_unique_noalloc(dummy, dummy, ctypes.c_uint32(limit + 1),
                                         ctypes.c_int32(32), ctypes.byref(count), None)
    assert rc == rw.RW_ERR_ARG
    rc = rw.lib().rw_tree_unique_noalloc(dummy, dummy, ctypes.c_uint32(0),
                                         ctypes.c_int32(32), ctypes.byref(count), None)
    assert rc == rw.RW_ERR_ARG


def test_noalloc_rejects_unaligned_or_overlapping_buffers(rw):
    """Host-side argument checks: the addresses below are never dereferenced,
    because both checks come before any device access."""
    count = ctypes.c_uint32(0)
    a, b = ctypes.c_void_p(1 << 20), ctypes.c_void_p(1 << 21)
    odd = ctypes.c_void_p((1 << 20) + 4)
    for key_bits in (32, 64):
        assert rw.lib().rw_tree_unique_noalloc(odd, b, ctypes.c_uint32(100),
                                               ctypes.c_int32(key_bits), ctypes.byref(count),
                                               None) == rw.RW_ERR_ARG
        assert rw.lib().rw_tree_unique_noalloc(a, odd, ctypes.c_uint32(100),
                                               ctypes.c_int32(key_bits), ctypes.byref(count),
                                               None) == rw.RW_ERR_ARG
    # in place, and overlapping by one key
    assert rw.lib().rw_tree_unique_noalloc(a, a, ctypes.c_uint32(100), ctypes.c_int32(32),
                                           ctypes.byref(count), None) == rw.RW_ERR_ARG
    near = ctypes.c_void_p((1 << 20) + 16 * 24)
    assert rw.lib().rw_tree_unique_noalloc(a, near, ctypes.c_uint32(100), ctypes.c_int32(32),
                                           ctypes.byref(count), None) == rw.RW_ERR_ARG
