"""GPU: the mixed-precision walks (FP64 offsets, FP32 interactions, FP64 sums)
against the FP64 forms of the same walk and against an FP64 direct sum.

Tolerances: the mixed result must agree with the plain FP64 result of the
same walk semantics to a median relative difference of 2e-6 (FP32 rounding
of ~thousands of terms summed in FP64 chunks) and its force error against the
FP64 direct sum must stay within 5% of the plain form's error."""
import numpy as np
import pytest

import pepc_b200 as P
from tests.datasets import cube, plummer

pytestmark = pytest.mark.gpu


def run(x, y, z, q, **kw):
    tc = P.TreeCode(**kw)
    g = tc.pepc_grow_tree(x, y, z, q)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    return tc, g, r


def relerr(r, d, idx):
    E = np.stack([r["ex"][idx], r["ey"][idx], r["ez"][idx]])
    Ed = np.stack([d["ex"], d["ey"], d["ez"]])
    return np.linalg.norm(E - Ed, axis=0) / np.linalg.norm(Ed, axis=0)


@pytest.mark.parametrize("walk,gs", [(P.WALK_GROUP, 64), (P.WALK_GROUP, 32),
                                     (P.WALK_PER_TARGET, 0), (P.WALK_PER_TILE, 0)])
def test_mixed_matches_plain_same_walk(gpu, walk, gs):
    x, y, z, q = plummer(60000, 41)
    kw = dict(theta2=0.16, eps2=1e-6, walk=walk, group_size=gs)
    tp, gp, rp = run(x, y, z, q, precision=P.PRECISION_PLAIN, **kw)
    tm, gm, rm = run(x, y, z, q, precision=P.PRECISION_MIXED, **kw)
    assert np.array_equal(gp.key, gm.key)
    idx = np.arange(0, 60000, 13)
    diff = relerr(rm, {"ex": rp["ex"][idx], "ey": rp["ey"][idx], "ez": rp["ez"][idx]}, idx)
    assert np.median(diff) < 2e-6, np.median(diff)
    assert np.percentile(diff, 99) < 1e-4
    pd = np.abs(rm["pot"] - rp["pot"]) / np.abs(rp["pot"])
    assert np.median(pd) < 2e-6
    # MAC decisions on FP32 offsets rarely flip: interaction counts agree almost everywhere
    assert np.mean(rm["work"] == rp["work"]) > 0.99
    d = tp.direct(idx)
    ep, em = relerr(rp, d, idx), relerr(rm, d, idx)
    assert np.median(em) <= 1.05 * np.median(ep) + 1e-7


def test_mixed_group_alternating_charges(gpu):
    # +-1 charges: strong cancellation, the hardest case for FP32 sums
    x, y, z, q = cube(40000, 42)
    kw = dict(theta2=0.09, eps2=1e-4, walk=P.WALK_GROUP, group_size=64)
    tp, _, rp = run(x, y, z, q, precision=P.PRECISION_PLAIN, **kw)
    tm, _, rm = run(x, y, z, q, precision=P.PRECISION_MIXED, **kw)
    idx = np.arange(0, 40000, 11)
    d = tp.direct(idx)
    ep, em = relerr(rp, d, idx), relerr(rm, d, idx)
    assert np.median(em) <= 1.05 * np.median(ep) + 1e-6
    st = tm.stats()
    assert st["interactions"] > 0 and st["twig_interactions"] > 0 and st["leaf_interactions"] > 0


def test_group_walk_work_counts(gpu):
    x, y, z, q = plummer(20000, 43)
    tm, _, rm = run(x, y, z, q, precision=P.PRECISION_MIXED, walk=P.WALK_GROUP, theta2=0.36)
    st = tm.stats()
    # every target's work counts its interactions (self included); the
    # library's leaf counter excludes the self term
    assert int(rm["work"].sum()) == st["leaf_interactions"] + st["twig_interactions"] + 20000


def test_mixed_group_periodic_matches_plain(gpu):
    # 27 mirror boxes walked inside the kernel, plus the lattice term
    rng = np.random.default_rng(44)
    n = 20000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    kw = dict(theta2=0.16, eps2=1e-4, walk=P.WALK_GROUP, periodicity=(1, 1, 1), group_size=64)
    _, _, rp = run(x, y, z, q, precision=P.PRECISION_PLAIN, **kw)
    _, _, rm = run(x, y, z, q, precision=P.PRECISION_MIXED, **kw)
    idx = np.arange(0, n, 7)
    diff = relerr(rm, {"ex": rp["ex"][idx], "ey": rp["ey"][idx], "ez": rp["ez"][idx]}, idx)
    # alternating charges cancel, so FP32 rounding shows more than for equal charges
    assert np.median(diff) < 2e-5, np.median(diff)
    assert np.mean(rm["work"] == rp["work"]) > 0.99


def test_mixed_group_ragged_buckets_and_duplicates(gpu):
    # N not a multiple of 32 (a partial last bucket) and coincident positions
    # (the duplicate-key fix moves them apart by less than the FP32 resolution
    # at the group scale, so the walk's exact FP64 self test is exercised)
    rng = np.random.default_rng(45)
    n = 4099
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    dup = rng.choice(n, 200, replace=False)
    x[dup[:100]], y[dup[:100]], z[dup[:100]] = x[dup[100:]], y[dup[100:]], z[dup[100:]]
    q = rng.standard_normal(n)
    kw = dict(theta2=0.25, eps2=1e-4, walk=P.WALK_GROUP, group_size=64)
    tp, gp, rp = run(x, y, z, q, precision=P.PRECISION_PLAIN, **kw)
    tm, gm, rm = run(x, y, z, q, precision=P.PRECISION_MIXED, **kw)
    assert np.array_equal(gp.key, gm.key)
    idx = np.arange(n)
    diff = relerr(rm, {"ex": rp["ex"], "ey": rp["ey"], "ez": rp["ez"]}, idx)
    assert np.median(diff) < 2e-5, np.median(diff)
    assert np.all(np.isfinite(rm["pot"]))
    assert np.mean(rm["work"] == rp["work"]) > 0.99


def test_mixed_group_bmax_mac_matches_plain(gpu):
    x, y, z, q = plummer(30000, 46)
    kw = dict(theta2=0.36, eps2=1e-6, walk=P.WALK_GROUP, mac_select=1, group_size=64)
    tp, _, rp = run(x, y, z, q, precision=P.PRECISION_PLAIN, **kw)
    tm, _, rm = run(x, y, z, q, precision=P.PRECISION_MIXED, **kw)
    idx = np.arange(0, 30000, 7)
    diff = relerr(rm, {"ex": rp["ex"][idx], "ey": rp["ey"][idx], "ez": rp["ez"][idx]}, idx)
    assert np.median(diff) < 2e-6, np.median(diff)
    assert np.mean(rm["work"] == rp["work"]) > 0.99
    # the Bmax MAC is the stricter one here: more interactions than Barnes-Hut
    _, _, rb = run(x, y, z, q, precision=P.PRECISION_MIXED, theta2=0.36, eps2=1e-6,
                   walk=P.WALK_GROUP)
    assert rm["work"].sum() != rb["work"].sum()


@pytest.mark.parametrize("data", ["plummer", "alternating"])
def test_mixed_strict_equals_fp64_group_lists(gpu, data):
    # the north star's precision form: FP64 offsets per interaction, Kahan-
    # compensated FP32 sums, and the FP64 group walk's MAC decisions, so every
    # target's interaction list (hence work and the counts) is the FP64 walk's
    if data == "plummer":
        x, y, z, q = plummer(60000, 43)
        kw = dict(theta2=0.16, eps2=1e-6, walk=P.WALK_GROUP, group_size=64)
    else:
        x, y, z, q = cube(40000, 44)
        kw = dict(theta2=0.09, eps2=1e-4, walk=P.WALK_GROUP, group_size=64)
    n = len(x)
    tp, gp, rp = run(x, y, z, q, precision=P.PRECISION_PLAIN, **kw)
    ts, gs_, rs = run(x, y, z, q, precision=P.PRECISION_MIXED_STRICT, **kw)
    tm, gm, rm = run(x, y, z, q, precision=P.PRECISION_MIXED, **kw)
    assert np.array_equal(rs["work"], rp["work"])
    sp, ss = tp.stats(), ts.stats()
    assert ss["twig_interactions"] == sp["twig_interactions"]
    # the FP64 walk counts each target's own leaf as an interaction, as the
    # reference does (module_tree_walk_pthreads.f90:617-631); the mixed walks
    # count only evaluated pairs
    assert ss["leaf_interactions"] + n == sp["leaf_interactions"]
    idx = np.arange(0, n, 13)
    ref = {"ex": rp["ex"][idx], "ey": rp["ey"][idx], "ez": rp["ez"][idx]}
    ds, dm = relerr(rs, ref, idx), relerr(rm, ref, idx)
    assert np.median(ds) < 2e-6 and np.percentile(ds, 99) < 1e-4
    # FP64 offsets and compensated sums are no less accurate than the default form
    assert np.median(ds) <= 1.05 * np.median(dm) + 1e-9
    d = tp.direct(idx)
    assert np.median(relerr(rs, d, idx)) <= 1.05 * np.median(relerr(rp, d, idx)) + 1e-7


def test_mixed_strict_only_for_the_64_target_group_walk(gpu):
    for kw in (dict(walk=P.WALK_PER_TARGET), dict(walk=P.WALK_GROUP, group_size=32)):
        with pytest.raises(P.PepcgError) as e:
            P.TreeCode(precision=P.PRECISION_MIXED_STRICT, **kw)
        assert e.value.code == P.PEPCG_ERR_UNSUPPORTED
