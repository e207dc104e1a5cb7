"""CPU tests: the oracle (a C++ restatement of the reference) is pinned to the
reference's own code and known answers, and its invariants hold."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.datasets import rocksalt

GOLD = os.path.join(os.path.dirname(__file__), "golden", "reference_pins.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def test_par_rand_kat(gold):
    # frontends/pepc-mini/module_helper.f90:586-590 documents the first draws
    r = O.par_rand(-1, 3)
    assert np.allclose(r, gold["par_rand_kat"], rtol=0, atol=5e-8)


@pytest.mark.parametrize("name", ["distinct", "dups", "large"])
def test_sort_matches_reference_sort(gold, name):
    # the golden permutation comes from the reference's sl_pepc sort_radix.c
    keys = gold[f"sort_{name}_in"]
    k, idx = O.sort_radix(keys)
    assert np.array_equal(idx, gold[f"sort_{name}_idx"].astype(np.int64))
    assert np.array_equal(k, keys[idx])


def test_sort_live_reference_if_built():
    if O.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(7)
    keys = rng.integers(1 << 60, 1 << 61, size=20000, dtype=np.int64)
    keys = keys[rng.integers(0, 20000, size=20000)]
    a = O.sort_radix(keys)
    b = O.ref_sort(keys)
    assert np.array_equal(a[1], b[1])


def test_lattice_coefficients_recompute_reference_table(gold):
    # the pretabulated unit-cube coefficients (module_fmm_framework.f90:260-508)
    # versus the oracle's restatement of calc_lattice_coefficients (:154-213)
    # at Lmax_multipole = 20: agreement to the truncation of the expansion
    p = O.params(periodicity=(1, 1, 1))
    ML = O.lattice_coefficients(p)
    tbl = lambda l, m: l * (l + 1) // 2 + m  # noqa: E731
    for l, m, v in zip(gold["lattice_l"], gold["lattice_m"], gold["lattice_v"]):
        if l > 40 or l < 4:
            continue
        assert abs(ML[tbl(l, m)].real - v) <= 1e-8 * abs(v)


def test_box_margin():
    x = np.array([0.0, 1.0, 0.5])
    y = np.array([2.0, 3.0, 2.5])
    z = np.array([-1.0, 1.0, 0.0])
    b = O.box_create(x, y, z)
    # module_box.f90:81-84
    for d, (lo, hi) in enumerate([(0.0, 1.0), (2.0, 3.0), (-1.0, 1.0)]):
        s = hi - lo
        assert b[d] == lo - s / 10000.0
        assert b[3 + d] == hi + s / 10000.0
        assert b[6 + d] == b[3 + d] - b[d]


def test_hilbert_keys_roundtrip():
    rng = np.random.default_rng(3)
    x, y, z = rng.random(500), rng.random(500), rng.random(500)
    b = O.box_create(x, y, z)
    k = O.compute_keys(x, y, z, b[:3], b[6:])
    assert np.all((k >> 60) == 1)  # placeholder bit at level 20
    # key_to_coord returns the centre of the key's cell: same key again
    for i in range(0, 500, 25):
        c = O.key_to_coord(k[i], b[:3], b[6:])
        k2 = O.compute_keys([c[0]], [c[1]], [c[2]], b[:3], b[6:])
        assert k2[0] == k[i]


def test_hilbert_adjacency():
    # consecutive Hilbert keys at level 20 are face neighbours
    rng = np.random.default_rng(4)
    b = np.array([0, 0, 0, 1, 1, 1, 1, 1, 1], dtype=float)
    base = rng.integers(1 << 60, (1 << 61) - 2, size=200, dtype=np.int64)
    s = 1.0 / (1 << 20)
    for k in base:
        c0 = O.key_to_coord(k, b[:3], b[6:])
        c1 = O.key_to_coord(k + 1, b[:3], b[6:])
        assert np.isclose(np.abs(c1 - c0).sum(), s)


def test_tree_invariants_and_walk_limits():
    rng = np.random.default_rng(5)
    n = 3000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    for walk in (0, 1):
        orc = O.Oracle(theta2=0.0, eps2=1e-4, walk=walk, num_threads=4)
        g = orc.grow_tree(x, y, z, q)
        t = orc.tree()
        # module_tree_grow.f90:97-105
        assert t["leaves"][0] == n
        nleaf = int(np.sum(t["descendants"] == 0))
        assert nleaf == n
        assert t["descendants"][0] + 1 == len(t["key"])
        r = orc.traverse_tree(g["x"], g["y"], g["z"], keys=g["key"])
        # theta = 0: every target interacts with every leaf (work = n)
        assert np.all(r["work"] == n)
        d = orc.direct(np.arange(0, n, 97))
        idx = np.arange(0, n, 97)
        rel = np.abs(r["ex"][idx] - d["ex"]) / np.abs(d["ex"]).max()
        assert rel.max() < 1e-12


def test_oracle_madelung_constant(gold):
    # rock-salt lattice in the periodic unit cube, all near-field boxes summed
    # directly (theta = 0) plus the reference's far-lattice term with its
    # pretabulated coefficients: -<q phi> r0 is the Madelung constant of NaCl
    n = 8
    x, y, z, q = rocksalt(n)
    orc = O.Oracle(theta2=0.0, eps2=0.0, periodicity=(1, 1, 1), num_threads=4)
    orc.set_lattice_coefficients(O.reference_lattice_table(gold))
    g = orc.grow_tree(x, y, z, q)
    r = orc.traverse_tree(g["x"], g["y"], g["z"])
    m_est = -np.mean(g["q"] * r["pot"]) / n
    assert abs(m_est - 1.7475645946331822) < 1e-8


def test_oracle_spatial_cutoff_zero_cuts_everything():
    # any(abs(delta) >= 0) holds for every node: no interaction is evaluated.
    # The pthreads walk still counts each leaf it reaches as work
    # (module_tree_walk_pthreads.f90:620-622); the simple walk counts nothing
    # (module_tree_walk_simple.f90:330,377)
    rng = np.random.default_rng(74)
    n = 500
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = rng.standard_normal(n)
    for walk in (0, 1):
        orc = O.Oracle(theta2=0.25, eps2=1e-4, walk=walk, spatial_interaction_cutoff=(0.0, 0.0, 0.0))
        g = orc.grow_tree(x, y, z, q)
        r = orc.traverse_tree(g["x"], g["y"], g["z"], keys=g["key"])
        assert not np.any(r["pot"]) and not np.any(r["ex"])
        assert orc.counters()["interactions"] == 0
        if walk == 0:
            assert np.all(r["work"] >= 1)
        else:
            assert not np.any(r["work"])
        orc.close()
