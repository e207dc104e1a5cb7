"""GPU: the device time-step pieces (push, external field, periodic wrap,
key-order gather) bit for bit against the oracle's restatement of the
pepc-mini frontend, and a device-resident multi-step loop against the same
loop on the oracle."""
import numpy as np
import pytest
import torch

import pepc_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda", 0)


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(DEV)


def H(t):
    return t.cpu().numpy()


def test_push_and_field_bitwise(gpu):
    rng = np.random.default_rng(71)
    n = 5000
    q, m = rng.standard_normal(n), rng.random(n) + 0.5
    e = [rng.standard_normal(n) for _ in range(3)]
    v = [rng.standard_normal(n) for _ in range(3)]
    x = [rng.random(n) for _ in range(3)]
    dv, dx = [T(a) for a in v], [T(a) for a in x]
    tc = P.TreeCode()
    tc.push_particles_device(1e-3, T(q), T(m), [T(a) for a in e], dv, dx)
    O.push_particles(1e-3, q, m, e, v, x)
    for a, b in zip(dv + dx, v + x):
        assert np.array_equal(H(a), b)
    ez, pot = rng.standard_normal(n), rng.standard_normal(n)
    dez, dpot = T(ez), T(pot)
    tc.apply_external_field_device(0.3, dx[2], dez, dpot)
    O.apply_external_field(0.3, x[2], ez, pot)
    assert np.array_equal(H(dez), ez) and np.array_equal(H(dpot), pot)
    tc.close()


@pytest.mark.parametrize("lattice", ["principal", "skewed"])
def test_wrap_bitwise(gpu, lattice):
    rng = np.random.default_rng(72)
    n = 5000
    c = [rng.uniform(-2.0, 3.0, n) for _ in range(3)]
    if lattice == "principal":
        kw = dict(periodicity=(1, 0, 1), t_lattice_1=(2.0, 0.0, 0.0), t_lattice_2=(0.0, 1.0, 0.0),
                  t_lattice_3=(0.0, 0.0, 0.5), lattice_origin=(0.1, -0.2, 0.0))
    else:
        kw = dict(periodicity=(1, 1, 1), t_lattice_1=(1.0, 0.0, 0.0), t_lattice_2=(0.5, 1.0, 0.0),
                  t_lattice_3=(0.0, 0.3, 1.0), include_far_field_if_periodic=0)
    dc = [T(a) for a in c]
    tc = P.TreeCode(**kw)
    tc.constrain_periodic_device(*dc)
    O.constrain_periodic(*c, **kw)
    for a, b in zip(dc, c):
        assert np.array_equal(H(a), b)
    tc.close()


def test_gather_follows_the_grow(gpu):
    rng = np.random.default_rng(73)
    n = 3000
    x, y, z, q = rng.random(n), rng.random(n), rng.random(n), rng.standard_normal(n)
    tc = P.TreeCode()
    g = tc.pepc_grow_tree(x, y, z, q)
    v = rng.standard_normal(n)
    out = torch.empty(n, dtype=torch.float64, device=DEV)
    tc.gather_device(T(v), out)
    assert np.array_equal(H(out), v[g.perm])
    with pytest.raises(P.PepcgError):
        src = T(v)
        tc.gather_device(src, src)
    tc.close()


def test_device_resident_steps_match_the_oracle_loop(gpu):
    # periodic (mirror boxes, no far field: bit-exact walks), three kick-drift
    # steps with the wrap; the particle state follows each grow's key order
    rng = np.random.default_rng(74)
    n = 2000
    kw = dict(theta2=0.25, eps2=1e-4, periodicity=(1, 1, 1), include_far_field_if_periodic=0)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    m = np.full(n, 1.0)
    dt = 2e-4
    # oracle loop on numpy
    ox, oy, oz, oq, om = x.copy(), y.copy(), z.copy(), q.copy(), m.copy()
    ov = [np.zeros(n) for _ in range(3)]
    orc = O.Oracle(walk=0, **kw)
    for _ in range(3):
        g = orc.grow_tree(ox, oy, oz, oq)
        p = g["perm"]
        ox, oy, oz, oq, om = g["x"].copy(), g["y"].copy(), g["z"].copy(), oq[p], om[p]
        ov = [a[p] for a in ov]
        r = orc.traverse_tree(ox, oy, oz, keys=g["key"])
        pos = [ox, oy, oz]
        O.push_particles(dt, oq, om, [r["ex"], r["ey"], r["ez"]], ov, pos)
        O.constrain_periodic(*pos, **kw)
    # device loop
    tc = P.TreeCode(walk=P.WALK_PER_TARGET, **kw)
    tc.set_stream(torch.cuda.current_stream().cuda_stream)
    dx, dy, dz, dq, dm = T(x), T(y), T(z), T(q), T(m)
    dv = [torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(3)]
    key = torch.empty(n, dtype=torch.int64, device=DEV)
    for _ in range(3):
        tc.grow_tree_device(dx, dy, dz, dq)
        nx, ny, nz, nq = (torch.empty(n, dtype=torch.float64, device=DEV) for _ in range(4))
        tc.particles_device(key, torch.empty(n, dtype=torch.int64, device=DEV), nx, ny, nz, nq)
        nm = torch.empty_like(dm)
        tc.gather_device(dm, nm)
        nv = [torch.empty_like(a) for a in dv]
        for a, b in zip(dv, nv):
            tc.gather_device(a, b)
        dx, dy, dz, dq, dm, dv = nx, ny, nz, nq, nm, nv
        out = [torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(5)]
        tc.traverse_self_device(*out)
        tc.push_particles_device(dt, dq, dm, out[:3], dv, [dx, dy, dz])
        tc.constrain_periodic_device(dx, dy, dz)
    torch.cuda.synchronize()
    for a, b in zip([dx, dy, dz] + dv, [ox, oy, oz] + ov):
        assert np.array_equal(H(a), b)
    tc.close()


@pytest.mark.parametrize("walk", [P.WALK_PER_TARGET, P.WALK_GROUP])
@pytest.mark.parametrize("precision", [P.PRECISION_PLAIN, P.PRECISION_MIXED])
def test_sharded_targets_equal_one_call(gpu, walk, precision):
    # three ranks' shares of the key-ordered targets, each walked alone, give
    # the single-call fields bit for bit (shares start at multiples of 32)
    rng = np.random.default_rng(75)
    n = 10007
    x, y, z, q = rng.random(n), rng.random(n), rng.random(n), rng.standard_normal(n)
    tc = P.TreeCode(theta2=0.25, eps2=1e-4, walk=walk, precision=precision)
    tc.grow_tree_device(T(x), T(y), T(z), T(q))
    full = [torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(5)]
    tc.traverse_self_device(*full)
    parts = [torch.zeros(n, dtype=torch.float64, device=DEV) for _ in range(5)]
    for r in range(3):
        t0, t1 = P.shard_range(n, r, 3)
        tc.traverse_range_device(t0, t1, *[p[t0:t1] for p in parts])
    for a, b in zip(full, parts):
        assert torch.equal(a, b)
    tc.close()


def test_sharded_tiles_follow_the_range_keys(gpu):
    # per-tile semantics on a share: tiles come from the share's own keys, as
    # they would from a rank's local keys; checked against the oracle
    rng = np.random.default_rng(76)
    n = 6000
    x, y, z, q = rng.random(n), rng.random(n), rng.random(n), rng.standard_normal(n)
    tc = P.TreeCode(theta2=0.25, eps2=1e-4, walk=P.WALK_PER_TILE)
    g = tc.pepc_grow_tree(x, y, z, q)
    orc = O.Oracle(theta2=0.25, eps2=1e-4, walk=1)
    go = orc.grow_tree(x, y, z, q)
    t0, t1 = P.shard_range(n, 1, 2)
    out = [torch.zeros(t1 - t0, dtype=torch.float64, device=DEV) for _ in range(5)]
    tc.traverse_range_device(t0, t1, *out)
    ro = orc.traverse_tree(go["x"][t0:t1], go["y"][t0:t1], go["z"][t0:t1], keys=go["key"][t0:t1])
    for k, a in zip(("ex", "ey", "ez", "pot", "work"), out):
        assert np.array_equal(H(a), ro[k]), k
    tc.close()


def test_restore_undoes_gather(gpu):
    rng = np.random.default_rng(77)
    n = 4000
    x, y, z, q = rng.random(n), rng.random(n), rng.random(n), rng.standard_normal(n)
    tc = P.TreeCode()
    tc.pepc_grow_tree(x, y, z, q)
    v = T(rng.standard_normal(n))
    a, b = torch.empty_like(v), torch.empty_like(v)
    tc.gather_device(v, a)
    tc.restore_device(a, b)
    assert torch.equal(b, v)
    tc.close()


def test_potential_energy_reduction(gpu):
    # pepc-b's potenergy (module_diagnostics.f90:227-263): sum of 0.5 q phi in
    # FP64, here on the device.  Against the exactly rounded sum (math.fsum) to
    # a few ulps of the magnitudes summed, the same value on repeated calls,
    # exact where every partial sum is exact, and 0 for no particles.
    import math
    rng = np.random.default_rng(77)
    x, y, z = rng.random(200000), rng.random(200000), rng.random(200000)
    q = rng.standard_normal(200000)
    tc = P.TreeCode(theta2=0.16, eps2=1e-4)
    g = tc.pepc_grow_tree(x, y, z, q)
    qd = T(q[g.perm])
    out = [torch.zeros(len(q), dtype=torch.float64, device=DEV) for _ in range(5)]
    tc.traverse_self_device(*out)
    pot = out[3]
    e1 = tc.potential_energy_device(qd, pot)
    e2 = tc.potential_energy_device(qd, pot)
    assert e1 == e2
    terms = (0.5 * H(qd)) * H(pot)
    exact = math.fsum(terms)
    assert abs(e1 - exact) <= 1e-15 * len(terms) * np.abs(terms).max()
    # small integers: every partial sum is exact, so the result is too
    qi = T(rng.integers(-8, 8, 100001).astype(np.float64))
    pi = T(rng.integers(-64, 64, 100001).astype(np.float64))
    assert tc.potential_energy_device(qi, pi) == math.fsum(0.5 * H(qi) * H(pi))
    assert tc.potential_energy_device(qi[:0], pi[:0]) == 0.0
    tc.close()
