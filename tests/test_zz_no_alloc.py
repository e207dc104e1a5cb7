"""GPU: pepcg_sort_keys_noalloc, the key sort for callers that cannot allocate
device memory (a frontend running inside another code's memory pool with
cudaMalloc forbidden, or one that must keep the device footprint fixed between
steps).  For distinct keys it must order them exactly as pepcg_grow_tree does
(equal keys keep their input order here): the tolerance is bit equality of the
sorted keys and of the permutation.

This file is collected last so that a run stopping at the first failure has
already run every other test; it passes alone in a fresh process as well."""
import ctypes as C

import numpy as np
import pytest

import pepc_b200 as P
from tests.datasets import cube, plummer

pytestmark = pytest.mark.gpu


def grown_order(x, y, z, q):
    """Keys in the caller's order, and the sorted keys and permutation that
    the existing entry point pepcg_grow_tree returns for them."""
    tc = P.TreeCode()
    g = tc.pepc_grow_tree(x, y, z, q)
    assert tc.stats()["dup_count"] == 0  # distinct keys: the order is unique
    keys_in = np.empty_like(g.key)
    keys_in[g.perm] = g.key
    tc.close()
    return keys_in, g.key, g.perm


def sort_noalloc(keys_in):
    import torch
    d_in = torch.from_numpy(keys_in).cuda()
    d_k = torch.full_like(d_in, -7)
    d_p = torch.full_like(d_in, -7)
    stream = torch.cuda.current_stream()
    rc = P.lib().pepcg_sort_keys_noalloc(len(keys_in), C.c_void_p(d_in.data_ptr()),
                                         C.c_void_p(d_k.data_ptr()), C.c_void_p(d_p.data_ptr()),
                                         C.c_void_p(stream.cuda_stream))
    assert rc == P.PEPCG_OK, P.lib().pepcg_last_error(None)
    torch.cuda.synchronize()
    return d_k.cpu().numpy(), d_p.cpu().numpy()


def test_noalloc_sort_matches_grow_order_twice(gpu):
    # two calls in a row; the second is smaller, so stale scratch contents
    # from the first call would show up in its result
    for n, seed, gen in ((300000, 61, cube), (70001, 62, plummer)):
        x, y, z, q = gen(n, seed)
        keys_in, key_ref, perm_ref = grown_order(x, y, z, q)
        k, p = sort_noalloc(keys_in)
        assert np.array_equal(k, key_ref)
        assert np.array_equal(p, perm_ref)


def test_noalloc_largest_size_allocates_nothing(gpu):
    # n = 2^20 fills the whole scratch layout (256 sort tiles and the full
    # histogram).  Equal keys keep their input order here, so the reference is
    # a stable sort of the keys as unsigned 64-bit values.  After a first call
    # (which looks up the scratch address and may load the library's kernels),
    # a second call must leave the device's free memory unchanged.
    import torch
    n = 1 << 20
    rng = np.random.default_rng(63)
    keys = rng.integers(1 << 60, 1 << 61, size=n // 2, dtype=np.int64)
    keys = keys[rng.integers(0, n // 2, size=n)]
    order = np.argsort(keys.view(np.uint64), kind="stable")
    k, p = sort_noalloc(keys)
    assert np.array_equal(p, order)
    assert np.array_equal(k, keys[order])
    d_in = torch.from_numpy(keys).cuda()
    d_k = torch.full_like(d_in, -7)
    d_p = torch.full_like(d_in, -7)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc = P.lib().pepcg_sort_keys_noalloc(n, C.c_void_p(d_in.data_ptr()), C.c_void_p(d_k.data_ptr()),
                                         C.c_void_p(d_p.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == P.PEPCG_OK, P.lib().pepcg_last_error(None)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert np.array_equal(d_p.cpu().numpy(), order)


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    rc = P.lib().pepcg_sort_keys_noalloc((1 << 20) + 1, None, None, None, None)
    assert rc == P.PEPCG_ERR_BAD_ARG
    assert b"1048576" in P.lib().pepcg_last_error(None)
