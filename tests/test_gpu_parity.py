"""GPU parity: libpepcg (through its C ABI) against the oracle on the same
seeded inputs.  Integer outputs (keys, order, tree structure, interaction
counts) must be identical; FP64 results of the plain form must be identical
too, because the device code evaluates the reference's expressions in the
reference's order without contraction (--fmad=false) and visits nodes in the
reference's order."""
import numpy as np
import pytest

import pepc_b200 as P
from oracle import oracle as O
from tests.datasets import cube, plummer

pytestmark = pytest.mark.gpu


def grow_both(x, y, z, q, **kw):
    tc = P.TreeCode(**kw)
    okw = {k: v for k, v in kw.items() if k in ("theta2", "eps2", "curve", "tile_size",
                                                  "periodicity", "force_cubic_domain",
                                                  "mac_select", "force_law",
                                                  "kelbg_invsqrttemp")}
    if "walk" in kw:
        okw["walk"] = 0 if kw["walk"] == P.WALK_PER_TARGET else 1
    orc = O.Oracle(num_threads=8, **okw)
    g = tc.pepc_grow_tree(x, y, z, q)
    go = orc.grow_tree(x, y, z, q)
    return tc, orc, g, go


@pytest.mark.parametrize("n,seed", [(2, 1), (3, 2), (17, 3), (1000, 4), (32768, 5)])
def test_grow_parity_uniform(gpu, n, seed):
    x, y, z, q = cube(n, seed)
    tc, orc, g, go = grow_both(x, y, z, q, theta2=0.36, eps2=1e-4)
    assert np.array_equal(g.key, go["key"])
    assert np.array_equal(g.perm, go["perm"])
    assert np.array_equal(g.x, go["x"]) and np.array_equal(g.y, go["y"]) and np.array_equal(g.z, go["z"])
    assert np.array_equal(tc.stats()["box"], orc.box())
    t, to = tc.tree(), orc.tree()
    for k in ("key", "level", "leaves", "descendants", "parent", "first_child", "next_sibling"):
        assert np.array_equal(t[k], to[k]), k
    assert np.array_equal(t["moments"], to["moments"])


def test_grow_parity_morton(gpu):
    x, y, z, q = cube(5000, 11)
    tc, orc, g, go = grow_both(x, y, z, q, curve=P.CURVE_MORTON)
    assert np.array_equal(g.key, go["key"])
    assert np.array_equal(g.perm, go["perm"])
    t, to = tc.tree(), orc.tree()
    assert np.array_equal(t["moments"], to["moments"])


def test_grow_parity_clustered(gpu):
    x, y, z, q = plummer(20000, 12)
    tc, orc, g, go = grow_both(x, y, z, q)
    assert np.array_equal(g.key, go["key"])
    assert np.array_equal(g.perm, go["perm"])
    t, to = tc.tree(), orc.tree()
    for k in ("key", "level", "leaves", "descendants", "parent"):
        assert np.array_equal(t[k], to[k]), k
    assert np.array_equal(t["moments"], to["moments"])


def test_grow_and_walk_deep_chain(gpu):
    # a tight cluster (spread 1e-6 of the box) under uniform background: long
    # chains of one-child twigs down to level 19-20, every level list non-empty
    x, y, z, q = cube(3000, 14, charges="gauss")
    rng = np.random.default_rng(15)
    c = np.array([0.3141, 0.5926, 0.5358])
    for i in range(40):
        x[i], y[i], z[i] = c + 1e-6 * rng.random(3)
    tc, orc, g, go = grow_both(x, y, z, q, theta2=0.16, eps2=1e-8, walk=P.WALK_PER_TARGET)
    assert tc.stats()["max_level"] >= 18
    assert np.array_equal(g.key, go["key"])
    t, to = tc.tree(), orc.tree()
    for k in ("key", "level", "leaves", "descendants", "parent"):
        assert np.array_equal(t[k], to[k]), k
    assert np.array_equal(t["moments"], to["moments"])
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k


@pytest.mark.parametrize("walk", [P.WALK_PER_TARGET, P.WALK_PER_TILE])
def test_force_cubic_domain_bit_exact(gpu, walk):
    # an elongated cloud: the cubic domain (module_box.f90:71-74) differs from
    # the bounding box, so keys, levels and MAC box lengths all change
    x, y, z, q = cube(6000, 16)
    x = 4.0 * x - 1.0
    z = 0.25 * z
    tc, orc, g, go = grow_both(x, y, z, q, theta2=0.36, eps2=1e-4, force_cubic_domain=1,
                               walk=walk, tile_size=16)
    assert np.array_equal(tc.stats()["box"], orc.box())
    assert np.array_equal(g.key, go["key"])
    assert np.array_equal(g.perm, go["perm"])
    t, to = tc.tree(), orc.tree()
    for k in ("key", "level", "leaves", "parent"):
        assert np.array_equal(t[k], to[k]), k
    assert np.array_equal(t["moments"], to["moments"])
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k
    # and the box is the cube, not the bounding box
    tb = P.TreeCode(theta2=0.36, eps2=1e-4)
    tb.pepc_grow_tree(x, y, z, q)
    assert not np.array_equal(tb.stats()["box"], tc.stats()["box"])


def test_grow_duplicate_positions(gpu):
    # duplicated positions give identical keys; the duplicate-key fix
    # (module_domains.f90:248-307) shifts keys and moves those particles
    x, y, z, q = cube(4000, 13)
    for a, b in [(10, 11), (500, 2000), (1234, 1235), (1234, 3999)]:
        x[b], y[b], z[b] = x[a], y[a], z[a]
    tc, orc, g, go = grow_both(x, y, z, q)
    assert tc.stats()["dup_count"] >= 3
    assert np.array_equal(g.key, go["key"])
    assert len(np.unique(g.key)) == len(g.key)
    assert np.array_equal(g.x, go["x"]) and np.array_equal(g.y, go["y"]) and np.array_equal(g.z, go["z"])
    # tied particles in the order of the reference's in-place MSD sort
    assert np.array_equal(g.perm, go["perm"])


@pytest.mark.parametrize("theta2", [0.0, 0.09, 0.36])
def test_walk_per_target_bit_exact(gpu, theta2):
    x, y, z, q = cube(20000, 21)
    tc, orc, g, go = grow_both(x, y, z, q, theta2=theta2, eps2=1e-4, walk=P.WALK_PER_TARGET)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k
    st = tc.stats()
    c = orc.counters()
    assert st["interactions"] == c["interactions"]
    assert st["mac_evaluations"] == c["mac_evaluations"]


@pytest.mark.parametrize("gs", [32, 64])
def test_walk_group_bit_exact(gpu, gs):
    # the group walk (buckets of gs key-consecutive targets, the simple walk's
    # rule) against the oracle's bucketed walk; 20,000 targets leave a ragged
    # last bucket
    x, y, z, q = plummer(20000, 17)
    tc = P.TreeCode(theta2=0.16, eps2=1e-6, walk=P.WALK_GROUP, group_size=gs)
    orc = O.Oracle(theta2=0.16, eps2=1e-6, walk=2, tile_size=gs, num_threads=8)
    g = tc.pepc_grow_tree(x, y, z, q)
    go = orc.grow_tree(x, y, z, q)
    assert np.array_equal(g.key, go["key"])
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k


@pytest.mark.parametrize("walk", [P.WALK_PER_TARGET, P.WALK_PER_TILE])
def test_walk_morton_keys_bit_exact(gpu, walk):
    x, y, z, q = plummer(8000, 29)
    tc, orc, g, go = grow_both(x, y, z, q, theta2=0.25, eps2=1e-4, walk=walk,
                               curve=P.CURVE_MORTON)
    assert np.array_equal(g.key, go["key"])
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k


@pytest.mark.parametrize("tile", [16, 32, 1, 7])
def test_walk_per_tile_bit_exact(gpu, tile):
    # tile sizes up to 16 run several tiles per warp (windows of 33 - T targets)
    x, y, z, q = cube(12000, 22, charges="gauss")
    tc, orc, g, go = grow_both(x, y, z, q, theta2=0.16, eps2=1e-6, walk=P.WALK_PER_TILE,
                               tile_size=tile)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k
    assert tc.stats()["interactions"] == orc.counters()["interactions"]
    assert tc.stats()["mac_evaluations"] == orc.counters()["mac_evaluations"]


@pytest.mark.parametrize("walk", [P.WALK_PER_TARGET, P.WALK_PER_TILE])
@pytest.mark.parametrize("mac", [1, 2])
def test_walk_other_macs_bit_exact(gpu, walk, mac):
    # mac_select 1: Bmax MAC, min(bmax^2, 3 boxlength2); 2: nothing accepted
    # (every target sees every particle, the N^2 code)
    n = 6000 if mac == 1 else 1500
    x, y, z, q = plummer(n, 25)
    tc, orc, g, go = grow_both(x, y, z, q, theta2=0.36, eps2=1e-6, walk=walk, mac_select=mac)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k
    assert tc.stats()["interactions"] == orc.counters()["interactions"]
    if mac == 2:
        assert np.all(r["work"] == n)  # every leaf, the self interaction included
        assert tc.stats()["twig_interactions"] == 0


@pytest.mark.parametrize("walk", [P.WALK_PER_TARGET, P.WALK_PER_TILE])
@pytest.mark.parametrize("law", [2, 4])
def test_walk_other_force_laws(gpu, walk, law):
    # force_law 2 (2D Coulomb: log potential, quadrupole in x, y) and 4
    # (Lennard-Jones quiet-start force); the walk is unchanged.  LJ uses only
    # + - * / sqrt, so it is bit-exact; the 2D law calls log, whose last bit
    # may differ between CUDA and the host library
    x, y, z, q = cube(6000, 26, charges="gauss")
    tc, orc, g, go = grow_both(x, y, z, q, theta2=0.25, eps2=1e-4, walk=walk, force_law=law)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    assert np.array_equal(r["work"], ro["work"])
    assert np.all(r["ez"] == 0.0) if law == 2 else np.all(r["pot"] == 0.0)
    for k in ("ex", "ey", "ez", "pot"):
        if law == 4:
            assert np.array_equal(r[k], ro[k]), k
        else:
            scale = np.abs(ro[k]).max() + 1e-300
            assert np.abs(r[k] - ro[k]).max() <= 1e-13 * scale, k
    d = tc.direct(np.arange(0, 6000, 97))
    do = orc.direct(np.arange(0, 6000, 97))
    for k in ("ex", "ey", "ez", "pot"):
        scale = np.abs(do[k]).max() + 1e-300
        assert np.abs(d[k] - do[k]).max() <= 1e-12 * scale, k


@pytest.mark.parametrize("walk", [P.WALK_PER_TARGET, P.WALK_PER_TILE])
def test_walk_kelbg(gpu, walk):
    # force_law 5: Kelbg leaves (erf / exp; lambda from the target's and the
    # source's charges) and unsoftened Coulomb twigs; the targets must be the
    # grown particles, whose charges the library knows
    x, y, z, q = cube(5000, 28)  # +1 / -1 alternating: e-i, i-i and e-e pairs
    kw = dict(theta2=0.25, eps2=1e-4, walk=walk, force_law=5, kelbg_invsqrttemp=20.0)
    tc, orc, g, go = grow_both(x, y, z, q, **kw)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    assert np.array_equal(r["work"], ro["work"])
    for k in ("ex", "ey", "ez", "pot"):
        scale = np.abs(ro[k]).max()
        assert np.abs(r[k] - ro[k]).max() <= 1e-13 * scale, k
    d = tc.direct(np.arange(0, 5000, 61))
    do = orc.direct(np.arange(0, 5000, 61))
    for k in ("ex", "ey", "ez", "pot"):
        scale = np.abs(do[k]).max()
        assert np.abs(d[k] - do[k]).max() <= 1e-12 * scale, k
    with pytest.raises(P.PepcgError) as ei:  # foreign targets: their charges are unknown
        tc.pepc_traverse_tree(np.array([0.5]), np.array([0.5]), np.array([0.5]))
    assert ei.value.code == P.PEPCG_ERR_UNSUPPORTED


def test_overwrite_results(gpu):
    # overwrite_results = 1: the old contents of ex..work are ignored, as if
    # the frontend had cleared them before the traverse
    x, y, z, q = cube(3000, 27)
    tc, orc, g, go = grow_both(x, y, z, q, theta2=0.25, eps2=1e-4, walk=P.WALK_PER_TARGET)
    r0 = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    tc.set_params(overwrite_results=1)
    junk = [np.full(3000, 7.0) for _ in range(3)]
    r1 = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key, e=junk, pot=np.full(3000, 5.0),
                               work=np.full(3000, 3.0))
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r0[k], r1[k]), k


def test_walk_accumulates_and_foreign_targets(gpu):
    x, y, z, q = plummer(15000, 23)
    tc, orc, g, go = grow_both(x, y, z, q, theta2=0.25, eps2=1e-6, walk=P.WALK_PER_TARGET)
    rng = np.random.default_rng(5)
    tx, ty, tz = rng.normal(size=300), rng.normal(size=300), rng.normal(size=300) * 3
    e0 = [rng.random(300), rng.random(300), rng.random(300)]
    p0, w0 = rng.random(300), np.ones(300)
    r = tc.pepc_traverse_tree(tx, ty, tz, e=e0, pot=p0, work=w0)
    ro = orc.traverse_tree(tx, ty, tz, e=e0, pot=p0, work=w0)
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k


def test_walk_per_tile_unkeyed_and_keyed_probes(gpu):
    x, y, z, q = cube(8000, 24)
    tc, orc, g, go = grow_both(x, y, z, q, theta2=0.36, eps2=1e-4, walk=P.WALK_PER_TILE)
    rng = np.random.default_rng(6)
    tx, ty, tz = rng.random(257), rng.random(257), rng.random(257)
    r = tc.pepc_traverse_tree(tx, ty, tz)           # unkeyed: one tile per target
    ro = orc.traverse_tree(tx, ty, tz)
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k
    sel = np.sort(rng.choice(8000, 700, replace=False))  # keyed subset: own tiles
    r = tc.pepc_traverse_tree(g.x[sel], g.y[sel], g.z[sel], keys=g.key[sel])
    ro = orc.traverse_tree(go["x"][sel], go["y"][sel], go["z"][sel], keys=go["key"][sel])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k


def test_direct_sum_matches_oracle(gpu):
    x, y, z, q = cube(6000, 31, charges="gauss")
    tc, orc, g, go = grow_both(x, y, z, q, eps2=1e-4)
    idx = np.arange(0, 6000, 37)
    d = tc.direct(idx)
    do = orc.direct(idx)
    for k in ("ex", "ey", "ez", "pot"):
        scale = np.abs(do[k]).max()
        assert np.abs(d[k] - do[k]).max() <= 1e-12 * scale, k


def test_scalar_backend_bit_exact(gpu):
    rng = np.random.default_rng(8)
    for _ in range(20):
        pos = rng.random(3)
        qv = rng.standard_normal()
        mp = P.multipole_from_particle(pos, qv)
        mo = np.zeros(15)
        O.lib().orc_multipole_from_particle(O.dp(pos), qv, O.dp(mo))
        assert np.array_equal(mp, mo)
        nc = int(rng.integers(1, 9))
        ch = rng.standard_normal((nc, 15))
        ch[:, 4] = np.abs(ch[:, 4])
        ch[:, 14] = np.abs(ch[:, 14])
        pp = P.shift_multipoles_up(ch)
        po = np.zeros(15)
        O.lib().orc_shift_multipoles_up(O.dp(po), O.dp(np.ascontiguousarray(ch)), nc)
        assert np.array_equal(pp, po)
        node = rng.standard_normal(15)
        dl = rng.standard_normal(3)
        d2 = float(dl @ dl)
        for fn, on in ((P.force_with_leaf, "orc_force_leaf"), (P.force_with_twig, "orc_force_twig")):
            e, ph = fn(node, dl, d2, 1e-3)
            eo, pho = np.zeros(3), np.zeros(1)
            getattr(O.lib(), on)(O.dp(node), O.dp(dl), d2 + 1e-3, O.dp(eo), O.dp(pho))
            assert np.array_equal(e, eo) and ph == pho[0]
    assert P.mac(0.36, 2.0, 0.5) and not P.mac(0.36, 1.0, 0.5)


def test_errors_are_reported(gpu):
    tc = P.TreeCode()
    with pytest.raises(P.PepcgError) as ei:
        tc.pepc_grow_tree([0.5], [0.5], [0.5], [1.0])
    assert ei.value.code == P.PEPCG_ERR_BAD_ARG
    x, y, z, q = cube(100, 9)
    x[7] = np.nan
    with pytest.raises(P.PepcgError) as ei:
        tc.pepc_grow_tree(x, y, z, q)
    assert ei.value.code == P.PEPCG_ERR_BAD_ARG
    # the failed grow's queued work (gather into key order) ends before the call
    # returns: the same context grows the corrected set like a fresh one
    x[7] = 0.25
    g = tc.pepc_grow_tree(x, y, z, q)
    go = O.Oracle().grow_tree(x, y, z, q)
    assert np.array_equal(g.key, go["key"]) and np.array_equal(g.perm, go["perm"])
    assert np.array_equal(g.x, go["x"])
    tc2 = P.TreeCode()
    with pytest.raises(P.PepcgError) as ei:
        tc2.pepc_traverse_tree([0.1], [0.1], [0.1])
    assert ei.value.code == P.PEPCG_ERR_NO_TREE
    with pytest.raises(P.PepcgError) as ei:
        P.TreeCode(force_law=6)
    assert ei.value.code == P.PEPCG_ERR_UNSUPPORTED
    with pytest.raises(P.PepcgError) as ei:
        P.TreeCode(force_law=2, precision=P.PRECISION_MIXED)
    assert ei.value.code == P.PEPCG_ERR_UNSUPPORTED
