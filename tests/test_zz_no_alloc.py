"""lumen_gpu_sort_pairs_noalloc, the sort entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc: code living inside a host
application that owns all device memory (an engine plugin, an FFI host with
its own allocator and budget) or a frame loop that must not allocate because
allocation can synchronise the device. Its work memory is a static device
array of the library, shared by every call.

The test calls it through the C ABI on caller-owned device buffers and
checks its result against the allocating entry point lumen_gpu_sort_pairs:
integer keys and indices must be identical (the same exact tolerance the
other sort tests use), on two calls in a row, so the second call also shows
that state left in the shared array by the first does not leak into it.
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _noalloc_sort(keys: np.ndarray, vals: np.ndarray):
    from lumen_b200 import _lib as L
    lib = L.load()
    k = torch.from_numpy(keys.view(np.int64).copy()).cuda()
    v = torch.from_numpy(vals.view(np.int32).copy()).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    status = lib.lumen_gpu_sort_pairs_noalloc(k.data_ptr(), v.data_ptr(), k.numel(), stream)
    return status, k.cpu().numpy().view(np.uint64), v.cpu().numpy().view(np.uint32)


def _reference_entry_point(keys: np.ndarray, vals: np.ndarray):
    from lumen_b200.render import sort_pairs
    k, v = sort_pairs(torch.from_numpy(keys.view(np.int64).copy()).cuda(),
                      torch.from_numpy(vals.view(np.int32).copy()).cuda())
    return k.cpu().numpy().view(np.uint64), v.cpu().numpy().view(np.uint32)


def _case(seed: int, n: int):
    rng = np.random.default_rng(seed)
    # tile-like upper half with many ties, depth-like lower half
    keys = (rng.integers(0, 500, size=n).astype(np.uint64) << np.uint64(32)) | \
        rng.integers(0, 20_000, size=n).astype(np.uint64)
    keys[::5] = keys[0]
    return keys, np.arange(n, dtype=np.uint32)


def test_noalloc_sort_matches_allocating_sort_twice():
    from lumen_b200 import _lib as L
    max_pairs = 262144   # LUMEN_GPU_NOALLOC_MAX_PAIRS in include/lumen_gpu.h
    for seed, n in ((1, 100_003), (2, max_pairs)):
        keys, vals = _case(seed, n)
        status, k, v = _noalloc_sort(keys, vals)
        assert status == L.LUMEN_SUCCESS, L.STATUS_NAMES.get(status, status)
        rk, rv = _reference_entry_point(keys, vals)
        assert np.array_equal(k, rk), "keys differ from lumen_gpu_sort_pairs"
        assert np.array_equal(v, rv), "permutation differs from lumen_gpu_sort_pairs"
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(v, order.astype(np.uint32))


@pytest.mark.parametrize("n", [1, 4095, 4096, 4097])
def test_noalloc_small_and_tile_edge_sizes_after_a_large_call(n):
    """Sizes inside one 4096-key tile and at its edge, each right after a
    full-size call, so the look-back descriptors and the alternate buffers
    that the large call left in the shared array are there to be misread.
    n = 1 has no varying digit: the pairs stay where the caller put them."""
    from lumen_b200 import _lib as L
    big_k, big_v = _case(3, 262144)
    assert _noalloc_sort(big_k, big_v)[0] == L.LUMEN_SUCCESS
    keys, vals = _case(10 + n, n)
    status, k, v = _noalloc_sort(keys, vals)
    assert status == L.LUMEN_SUCCESS
    rk, rv = _reference_entry_point(keys, vals)
    assert np.array_equal(k, rk) and np.array_equal(v, rv)
    assert np.array_equal(v, np.argsort(keys, kind="stable").astype(np.uint32))


def test_noalloc_all_equal_keys_after_a_large_call():
    """Every key equal (no digit varies): the order is the input order."""
    from lumen_b200 import _lib as L
    big_k, big_v = _case(4, 200_000)
    assert _noalloc_sort(big_k, big_v)[0] == L.LUMEN_SUCCESS
    for n in (4097, 100_000):
        keys = np.full(n, (7 << 32) | 12345, np.uint64)
        vals = np.arange(n, dtype=np.uint32)[::-1].copy()
        status, k, v = _noalloc_sort(keys, vals)
        assert status == L.LUMEN_SUCCESS
        assert np.array_equal(k, keys) and np.array_equal(v, vals)
        rk, rv = _reference_entry_point(keys, vals)
        assert np.array_equal(k, rk) and np.array_equal(v, rv)


def test_noalloc_rejects_sizes_beyond_the_static_array():
    from lumen_b200 import _lib as L
    lib = L.load()
    n = 262144 + 1
    k = torch.zeros(n, dtype=torch.int64, device="cuda")
    v = torch.zeros(n, dtype=torch.int32, device="cuda")
    status = lib.lumen_gpu_sort_pairs_noalloc(k.data_ptr(), v.data_ptr(), n, torch.cuda.current_stream().cuda_stream)
    assert status == -1   # LUMEN_ERROR_INVALID_ARGUMENT
