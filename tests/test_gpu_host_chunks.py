"""GPU: the host-array entry points overlap their transfers with the device
work -- pepcg_grow_tree copies its outputs back while the tree build and the
upward pass run, and pepcg_traverse_tree walks large target sets in three
chunks whose uploads and downloads overlap the walk.  The results must be
exactly those of the device entry points on the same particles, for every
walk that is split (per-target and group, plain and mixed), with and without
overwrite_results."""
import numpy as np
import pytest
import torch

import pepc_b200 as P

pytestmark = pytest.mark.gpu
N = 300000  # above the chunking threshold (262,144 targets)


def device_fields(tc, x, y, z, q, init=0.0):
    dev = torch.device("cuda", 0)
    tc.set_stream(torch.cuda.current_stream().cuda_stream)  # ordered with the torch fills
    tc.grow_tree_device(*(torch.from_numpy(a).to(dev) for a in (x, y, z, q)))
    out = [torch.full((len(x),), init, dtype=torch.float64, device=dev) for _ in range(5)]
    tc.traverse_self_device(*out)
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in out]


@pytest.mark.parametrize("precision,walk", [(P.PRECISION_MIXED, P.WALK_GROUP),
                                            (P.PRECISION_MIXED, P.WALK_PER_TARGET),
                                            (P.PRECISION_PLAIN, P.WALK_GROUP),
                                            (P.PRECISION_PLAIN, P.WALK_PER_TARGET)])
@pytest.mark.parametrize("overwrite", [0, 1])
def test_chunked_host_traverse_equals_device_path(gpu, precision, walk, overwrite):
    rng = np.random.default_rng(17)
    x, y, z = rng.random(N), rng.random(N), rng.random(N)
    q = np.where(np.arange(N) % 2 == 0, 1.0, -1.0) / N
    kw = dict(theta2=0.36 if precision == P.PRECISION_PLAIN else 0.16, eps2=1e-6,
              precision=precision, walk=walk)
    tc = P.TreeCode(overwrite_results=overwrite, **kw)
    # the walk adds onto the old results (1.0 everywhere), which overwrite_results
    # replaces by zeros
    ref = device_fields(tc, x, y, z, q, init=0.0 if overwrite else 1.0)
    g = tc.pepc_grow_tree(x, y, z, q)
    # the grown particles as targets, in key order: the fields of the device path
    ones = [np.ones(N) for _ in range(5)]
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key, e=ones[:3], pot=ones[3], work=ones[4])
    for k, name in enumerate(("ex", "ey", "ez", "pot", "work")):
        assert np.array_equal(r[name], ref[k]), name
    tc.close()


def test_chunked_host_traverse_ragged_count(gpu):
    """A target count that is not a multiple of 32: the last chunk is ragged."""
    n = 262144 + 1001
    rng = np.random.default_rng(19)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = rng.standard_normal(n) / n
    tc = P.TreeCode(theta2=0.16, eps2=1e-6, precision=P.PRECISION_MIXED, walk=P.WALK_GROUP,
                    overwrite_results=1)
    ref = device_fields(tc, x, y, z, q)
    g = tc.pepc_grow_tree(x, y, z, q)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    for k, name in enumerate(("ex", "ey", "ez", "pot", "work")):
        assert np.array_equal(r[name], ref[k]), name
    tc.close()


def test_host_grow_outputs_and_a_following_traverse(gpu):
    """Grow returns while the upward pass may still run; the next traverse is
    stream-ordered after it."""
    rng = np.random.default_rng(18)
    x, y, z = rng.random(N), rng.random(N), rng.random(N)
    q = rng.standard_normal(N) / N
    tc = P.TreeCode(theta2=0.16, eps2=1e-6, precision=P.PRECISION_MIXED, walk=P.WALK_GROUP)
    ref = device_fields(tc, x, y, z, q)
    dev = torch.device("cuda", 0)
    keys = torch.zeros(N, dtype=torch.int64, device=dev)
    perm = torch.zeros(N, dtype=torch.int64, device=dev)
    xs = [torch.zeros(N, dtype=torch.float64, device=dev) for _ in range(4)]
    tc.particles_device(keys, perm, *xs)
    torch.cuda.synchronize()
    for rep in range(3):
        g = tc.pepc_grow_tree(x, y, z, q)
        assert np.array_equal(g.key, keys.cpu().numpy())
        assert np.array_equal(g.perm, perm.cpu().numpy())
        assert np.array_equal(g.x, xs[0].cpu().numpy())
        r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
        for k, name in enumerate(("ex", "ey", "ez", "pot", "work")):
            assert np.array_equal(r[name], ref[k]), (rep, name)
    tc.close()
