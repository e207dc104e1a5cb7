"""GPU: the local key sort in the reference's order, equal keys included.

pepcg_sort_keys (and the sort inside pepcg_grow_tree) must return the
permutation of the reference's own sort (sl_pepc sort_radix.c, an in-place MSD
radix sort whose exchanges decide the order of equal keys).  The golden
permutations in tests/golden/reference_pins.npz were produced by that sort,
compiled from the reference's sources; larger cases compare with the oracle's
restatement of it, which the same fixtures pin.  The bar is bit equality."""
import os

import numpy as np
import pytest

import pepc_b200 as P
from oracle import oracle as O
from tests.datasets import cube

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "reference_pins.npz")


@pytest.fixture(scope="module")
def tc(gpu):
    t = P.TreeCode()
    yield t
    t.close()


@pytest.mark.parametrize("name", ["distinct", "dups", "large"])
def test_sort_keys_equals_reference_permutation(tc, name):
    gold = np.load(GOLD)
    keys = gold[f"sort_{name}_in"]
    k, p = tc.sort_keys(keys)
    assert np.array_equal(p, gold[f"sort_{name}_idx"].astype(np.int64))
    assert np.array_equal(k, keys[p])


def heavy_dups(n, seed, distinct):
    rng = np.random.default_rng(seed)
    base = rng.integers(1 << 60, 1 << 61, size=distinct, dtype=np.int64)
    return base[rng.integers(0, distinct, size=n)]


@pytest.mark.parametrize("n,distinct,seed", [(2, 1, 1), (3, 2, 2), (257, 40, 3), (5000, 5000, 4),
                                             (100000, 3000, 5), (300000, 290000, 6)])
def test_sort_keys_ties_match_oracle(tc, n, distinct, seed):
    keys = heavy_dups(n, seed, distinct)
    k, p = tc.sort_keys(keys)
    ko, po = O.sort_radix(keys)
    assert np.array_equal(p, po)
    assert np.array_equal(k, ko)


def test_sort_keys_deep_recursion(tc):
    # keys in a narrow range share the top digits: every class pass down to the
    # last digit (bits 3..0) runs on ranges of more than 256 elements
    rng = np.random.default_rng(9)
    keys = (np.int64(1) << 60) + rng.integers(0, 40, size=60000, dtype=np.int64)
    keys[::7] = (np.int64(1) << 60) + 17
    k, p = tc.sort_keys(keys)
    assert np.array_equal(p, O.sort_radix(keys)[1])
    one = np.full(5000, (1 << 60) + 12345, dtype=np.int64)
    assert np.array_equal(tc.sort_keys(one)[1], O.sort_radix(one)[1])


def test_sort_keys_device_and_sizes(tc):
    import torch
    keys = heavy_dups(70001, 12, 20000)
    d = torch.from_numpy(keys).cuda()
    ko = torch.empty_like(d)
    po = torch.empty_like(d)
    tc.sort_keys_device(d, ko, po)
    torch.cuda.synchronize()
    assert np.array_equal(po.cpu().numpy(), O.sort_radix(keys)[1])
    # empty and single-key calls
    assert tc.sort_keys(np.zeros(0, np.int64))[1].size == 0
    assert np.array_equal(tc.sort_keys(np.array([5], np.int64))[1], [0])


def test_grow_ties_in_reference_order(gpu):
    # many particles at shared positions: the tie order decides which particle
    # of each group gets a shifted key and new coordinates (module_domains.f90:
    # 276-307), and therefore every field
    x, y, z, q = cube(30000, 31, charges="normal")
    rng = np.random.default_rng(32)
    src = rng.integers(0, 30000, size=6000)
    dst = rng.integers(0, 30000, size=6000)
    x[dst], y[dst], z[dst] = x[src], y[src], z[src]
    tc = P.TreeCode(theta2=0.36, eps2=1e-4)
    orc = O.Oracle(theta2=0.36, eps2=1e-4, num_threads=8)
    g = tc.pepc_grow_tree(x, y, z, q)
    go = orc.grow_tree(x, y, z, q)
    assert tc.stats()["dup_count"] > 1000
    assert np.array_equal(g.perm, go["perm"])
    assert np.array_equal(g.key, go["key"])
    for a, b in ((g.x, go["x"]), (g.y, go["y"]), (g.z, go["z"])):
        assert np.array_equal(a, b)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k
    tc.close()
    orc.close()
