"""GPU: walks and adjoints of two contexts running at the same time on one
device, each context on its own stream and host thread, give the results each
context gives alone (the persistent kernels take their buckets from a counter
in their context's own memory).  Walk fields must match bit for bit; adjoint
gradients to 1e-10 relative."""
import threading

import numpy as np
import pytest

import pepc_b200 as P
from tests.datasets import cube, plummer

pytestmark = pytest.mark.gpu


def concurrently(*fns):
    out, errs = [None] * len(fns), []

    def run(i, f):
        try:
            out[i] = f()
        except Exception as e:  # noqa: BLE001 -- re-raised below
            errs.append(e)

    th = [threading.Thread(target=run, args=(i, f)) for i, f in enumerate(fns)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]
    return out


def test_two_contexts_walk_concurrently(gpu):
    xa, ya, za, qa = plummer(200000, 71)
    xb, yb, zb, qb = cube(150000, 72)
    ta = P.TreeCode(theta2=0.16, eps2=1e-6, walk=P.WALK_PER_TARGET)
    tb = P.TreeCode(theta2=0.16, eps2=1e-6, walk=P.WALK_GROUP, precision=P.PRECISION_MIXED)
    ga = ta.pepc_grow_tree(xa, ya, za, qa)
    gb = tb.pepc_grow_tree(xb, yb, zb, qb)
    walk_a = lambda: ta.pepc_traverse_tree(ga.x, ga.y, ga.z, keys=ga.key)  # noqa: E731
    walk_b = lambda: tb.pepc_traverse_tree(gb.x, gb.y, gb.z, keys=gb.key)  # noqa: E731
    alone_a, alone_b = walk_a(), walk_b()
    for _ in range(4):
        ra, rb = concurrently(walk_a, walk_b)
        for k in ("ex", "ey", "ez", "pot", "work"):
            assert np.array_equal(ra[k], alone_a[k]), k
            assert np.array_equal(rb[k], alone_b[k]), k
    ta.close()
    tb.close()


def test_two_contexts_adjoint_concurrently(gpu):
    rng = np.random.default_rng(73)
    res = []
    for seed in (74, 75):
        x, y, z, _ = cube(60000, seed)
        q = rng.standard_normal(60000)
        tc = P.TreeCode(theta2=0.16, eps2=1e-6, walk=P.WALK_PER_TARGET)
        tc.pepc_grow_tree(x, y, z, q)
        tx, ty, tz = (rng.random(2048) for _ in range(3))
        g = [rng.standard_normal(2048) for _ in range(4)]
        res.append((tc, lambda tc=tc, a=(tx, ty, tz, g[:3], g[3], 60000):
                    tc.traverse_adjoint(*a)))
    alone = [f() for _, f in res]
    for _ in range(4):
        both = concurrently(*(f for _, f in res))
        # the adjoint adds its records with atomics, so the sums' order (and
        # their last bits) may differ from run to run; a bucket walked twice or
        # not at all would differ at O(1)
        for got, ref in zip(both, alone):
            for k in ref:
                scale = np.abs(ref[k]).max()
                assert np.allclose(got[k], ref[k], rtol=1e-10, atol=1e-12 * scale), k
    for tc, _ in res:
        tc.close()
