"""GPU: the adjoint walk (pepcg_traverse_adjoint) -- dL/dq and dL/dx of the
sources for dL/dE and dL/dphi given at the targets.

Checks, all in FP64:
  * against the oracle's adjoint (same walk semantics, fixed lists):
    relative 1e-9 of the gradient's scale (atomic summation order differs);
  * against central finite differences of the GPU forward pass (h = 1e-6,
    the whole grow + traverse re-run per point): relative 1e-5, allowing a
    coordinate whose perturbation flips a MAC decision or a key;
  * force_law 2 (2D Coulomb) and 4 (Lennard-Jones) against the oracle and FD;
  * periodic boundaries with the FMM lattice term (each extrinsic
    correction): against the oracle, whose lattice adjoint differentiates the
    harmonics independently, and FD;
  * the adjoint configuration -- 262,144 sources U[0,1)^3 with q ~ N(0,1),
    4,096 probes U[0.25,0.75]^3, L = sum (phi - phi_target)^2 with
    phi_target from a second charge set, theta = 0.4, eps = 1e-3 -- against
    the FP64 direct-sum gradient (tree-code accuracy) and FD on 64 random
    coordinates."""
import os

import numpy as np
import pytest
import torch

import pepc_b200 as P
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.npz"))


def forward_L(x, y, z, q, tx, ty, tz, gphi, gE, **kw):
    tc = P.TreeCode(precision=P.PRECISION_PLAIN, **kw)
    tc.pepc_grow_tree(x, y, z, q)
    r = tc.pepc_traverse_tree(tx, ty, tz)
    tc.close()
    return float(np.sum(gphi * r["pot"] + gE[0] * r["ex"] + gE[1] * r["ey"] + gE[2] * r["ez"]))


def problem(n, nt, seed):
    rng = np.random.default_rng(seed)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = rng.standard_normal(n)
    tx, ty, tz = (0.25 + 0.5 * rng.random(nt) for _ in range(3))
    gphi = rng.standard_normal(nt)
    gE = [rng.standard_normal(nt) for _ in range(3)]
    return x, y, z, q, tx, ty, tz, gphi, gE, rng


@pytest.mark.parametrize("walk,mac", [(P.WALK_PER_TARGET, 0), (P.WALK_GROUP, 0),
                                      (P.WALK_PER_TARGET, 1)])
def test_adjoint_matches_oracle_and_fd(gpu, walk, mac):
    x, y, z, q, tx, ty, tz, gphi, gE, rng = problem(3000, 70, 71)
    kw = dict(theta2=0.16, eps2=1e-3, walk=walk, mac_select=mac)
    tc = P.TreeCode(precision=P.PRECISION_PLAIN, **kw)
    tc.pepc_grow_tree(x, y, z, q)
    g = tc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    if walk == P.WALK_PER_TARGET:
        orc = O.Oracle(theta2=0.16, eps2=1e-3, walk=0, mac_select=mac)
        orc.grow_tree(x, y, z, q)
        go = orc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
        for k in ("q", "x", "y", "z"):
            scale = np.abs(go[k]).max()
            assert np.abs(g[k] - go[k]).max() <= 1e-9 * scale, k
    h = 1e-6
    bad = 0
    for trial in range(16):
        j = int(rng.integers(len(x)))
        key = "xyzq"[trial % 4]
        arrs = {"x": x, "y": y, "z": z, "q": q}
        plus = {k: v.copy() for k, v in arrs.items()}
        minus = {k: v.copy() for k, v in arrs.items()}
        plus[key][j] += h
        minus[key][j] -= h
        fd = (forward_L(plus["x"], plus["y"], plus["z"], plus["q"], tx, ty, tz, gphi, gE, **kw) -
              forward_L(minus["x"], minus["y"], minus["z"], minus["q"], tx, ty, tz, gphi, gE, **kw)) / (2 * h)
        an = g[key][j]
        if abs(fd - an) > 1e-5 * max(abs(fd), abs(an), 1e-8):
            bad += 1
    assert bad <= 1


def test_adjoint_configuration_against_direct_and_fd(gpu):
    n, nt = 262144, 4096
    rng = np.random.default_rng(4)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = np.random.default_rng(41).standard_normal(n)
    prng = np.random.default_rng(42)
    tx, ty, tz = (0.25 + 0.5 * prng.random(nt) for _ in range(3))
    q_t = np.random.default_rng(43).standard_normal(n)
    kw = dict(theta2=0.16, eps2=1e-6, walk=P.WALK_PER_TARGET)
    # phi_target: the potential of the second charge set at the probes
    tt = P.TreeCode(precision=P.PRECISION_PLAIN, **kw)
    tt.pepc_grow_tree(x, y, z, q_t)
    phi_t = tt.pepc_traverse_tree(tx, ty, tz)["pot"]
    tt.close()
    tc = P.TreeCode(precision=P.PRECISION_PLAIN, **kw)
    tc.pepc_grow_tree(x, y, z, q)
    phi = tc.pepc_traverse_tree(tx, ty, tz)["pot"]
    gphi = 2.0 * (phi - phi_t)
    zero = [np.zeros(nt)] * 3
    g = tc.traverse_adjoint(tx, ty, tz, zero, gphi, n)
    # FP64 direct-sum gradient (no tree), oracle
    orc = O.Oracle(theta2=0.16, eps2=1e-6, walk=0, num_threads=16)
    orc.grow_tree(x, y, z, q)
    gd = orc.traverse_adjoint(tx, ty, tz, zero, gphi, n, direct=True)
    for k in ("q", "x"):
        rel = np.abs(g[k] - gd[k]) / np.abs(gd[k]).max()
        assert np.median(rel) < 1e-3, (k, np.median(rel))
    # central differences of L = sum (phi - phi_t)^2 on 64 random coordinates
    def L(xx, yy, zz, qq):
        t = P.TreeCode(precision=P.PRECISION_PLAIN, **kw)
        t.pepc_grow_tree(xx, yy, zz, qq)
        p = t.pepc_traverse_tree(tx, ty, tz)["pot"]
        t.close()
        return float(np.sum((p - phi_t) ** 2))
    h = 1e-6
    crng = np.random.default_rng(44)
    bad = 0
    for trial in range(64):
        j = int(crng.integers(n))
        key = "xyzq"[int(crng.integers(4))]
        arrs = {"x": x, "y": y, "z": z, "q": q}
        plus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        minus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        plus[key][j] += h
        minus[key][j] -= h
        fd = (L(plus["x"], plus["y"], plus["z"], plus["q"]) -
              L(minus["x"], minus["y"], minus["z"], minus["q"])) / (2 * h)
        an = g[key][j]
        if abs(fd - an) > 1e-4 * max(abs(fd), abs(an)) + 1e-9:
            bad += 1
    assert bad <= 3, bad


class TreeField(torch.autograd.Function):
    """phi, E at fixed probes as a function of the sources (x, y, z, q), with
    the backward pass through pepcg_traverse_adjoint_device.  Test harness
    only: the library itself has no torch dependency."""

    @staticmethod
    def forward(ctx, x, y, z, q, probes, tc):
        tc.grow_tree_device(x, y, z, q)
        tx, ty, tz = probes
        out = [torch.zeros_like(tx) for _ in range(5)]
        tc.traverse_tree_device(tx, ty, tz, *out)
        ctx.tc, ctx.probes, ctx.n = tc, probes, x.numel()
        return out[3], out[0], out[1], out[2]

    @staticmethod
    def backward(ctx, gphi, gex, gey, gez):
        tx, ty, tz = ctx.probes
        dev = tx.device
        g = [torch.zeros(ctx.n, dtype=torch.float64, device=dev) for _ in range(4)]
        z = torch.zeros_like(tx)
        gphi = gphi.contiguous() if gphi is not None else z
        gE = [a.contiguous() if a is not None else z for a in (gex, gey, gez)]
        ctx.tc.traverse_adjoint_device(tx, ty, tz, gE, gphi, *g)
        return g[1], g[2], g[3], g[0], None, None


def direct_grad_torch(x, y, z, q, tx, ty, tz, gphi, chunk=256):
    """FP64 direct-sum dL/dq, dL/dx for dL/dphi = gphi (torch, chunked)."""
    dq = torch.zeros_like(q)
    dx, dy, dz = torch.zeros_like(x), torch.zeros_like(x), torch.zeros_like(x)
    for s in range(0, tx.numel(), chunk):
        e = slice(s, s + chunk)
        rx = tx[e, None] - x[None, :]
        ry = ty[e, None] - y[None, :]
        rz = tz[e, None] - z[None, :]
        rinv = torch.rsqrt(rx * rx + ry * ry + rz * rz + 1e-6)
        g = gphi[e, None]
        dq += (g * rinv).sum(0)
        w = g * q[None, :] * rinv ** 3
        dx += (w * rx).sum(0)
        dy += (w * ry).sum(0)
        dz += (w * rz).sum(0)
    return dq, dx, dy, dz


def test_autograd_harness_against_torch_direct_gradient(gpu):
    """L = sum (phi - phi_t)^2 through torch.autograd with the adjoint as the
    backward; the gradient is compared with the FP64 direct-sum gradient in
    torch (tree accuracy at theta = 0.4)."""
    dev = torch.device("cuda", 0)
    n, nt = 65536, 1024
    rng = np.random.default_rng(8)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    x, y, z = (T(rng.random(n)) for _ in range(3))
    q = T(rng.standard_normal(n))
    probes = tuple(T(0.25 + 0.5 * rng.random(nt)) for _ in range(3))
    phi_t = T(rng.standard_normal(nt))
    tc = P.TreeCode(theta2=0.16, eps2=1e-6, precision=P.PRECISION_PLAIN, walk=P.WALK_GROUP)
    tc.set_stream(torch.cuda.current_stream().cuda_stream)
    leaves = [a.clone().requires_grad_(True) for a in (x, y, z, q)]
    phi, ex, ey, ez = TreeField.apply(*leaves, probes, tc)
    L = ((phi - phi_t) ** 2).sum()
    L.backward()
    gphi = 2.0 * (phi.detach() - phi_t)
    dq, dx, dy, dz = direct_grad_torch(x, y, z, q, *probes, gphi)
    for name, a, b in (("q", leaves[3].grad, dq), ("x", leaves[0].grad, dx),
                       ("y", leaves[1].grad, dy), ("z", leaves[2].grad, dz)):
        rel = ((a - b).abs() / b.abs().max()).cpu().numpy()
        assert np.median(rel) < 1e-3, (name, np.median(rel))
    tc.close()


@pytest.mark.parametrize("law", [2, 4])
@pytest.mark.parametrize("walk,owalk", [(P.WALK_PER_TARGET, 0), (P.WALK_GROUP, 2)])
def test_adjoint_other_force_laws(gpu, law, walk, owalk):
    """force_law 2 (2D Coulomb) and 4 (Lennard-Jones): the GPU adjoint differentiates
    the forward kernels by forward-mode dual numbers (D3), the oracle by the complex
    step.  GPU against oracle to 1e-9 of each component's scale (per-target and
    32-target bucket lists), then FD of the GPU forward to 1e-6 of that scale."""
    x, y, z, q, tx, ty, tz, gphi, gE, rng = problem(3000, 70, 90 + law)
    kw = dict(theta2=0.16, eps2=1e-3, force_law=law)
    tc = P.TreeCode(precision=P.PRECISION_PLAIN, walk=walk, group_size=32, **kw)
    tc.pepc_grow_tree(x, y, z, q)
    g = tc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    orc = O.Oracle(walk=owalk, tile_size=32, num_threads=8, **kw)
    orc.grow_tree(x, y, z, q)
    go = orc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    orc.close()
    for k in ("q", "x", "y", "z"):
        scale = np.abs(go[k]).max()
        if law == 2 and k == "z":  # the 2D law reads no z offsets
            assert np.abs(g[k]).max() <= 1e-12 * np.abs(go["x"]).max()
            continue
        assert np.abs(g[k] - go[k]).max() <= 1e-9 * scale, (k, scale)
    if walk != P.WALK_PER_TARGET:
        tc.close()
        return

    def L(a):
        tc.pepc_grow_tree(a["x"], a["y"], a["z"], a["q"])
        r = tc.pepc_traverse_tree(tx, ty, tz)
        return float(np.sum(gphi * r["pot"] + gE[0] * r["ex"] + gE[1] * r["ey"] + gE[2] * r["ez"]))

    h = 1e-5
    for trial in range(12):
        j = int(rng.integers(len(x)))
        key = "xyq"[trial % 3]
        arrs = {"x": x, "y": y, "z": z, "q": q}
        plus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        minus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        plus[key][j] += h
        minus[key][j] -= h
        fd = (L(plus) - L(minus)) / (2 * h)
        assert abs(fd - g[key][j]) <= 1e-6 * np.abs(g[key]).max(), (key, j, fd, g[key][j])
    tc.close()


def test_adjoint_refuses_kelbg(gpu):
    x, y, z, q, tx, ty, tz, gphi, gE, rng = problem(500, 8, 94)
    tc = P.TreeCode(precision=P.PRECISION_PLAIN, force_law=5, kelbg_invsqrttemp=1.0, eps2=0.0)
    tc.pepc_grow_tree(x, y, z, np.where(np.arange(500) % 2 == 0, 1.0, -1.0))
    with pytest.raises(P.PepcgError) as e:
        tc.traverse_adjoint(tx, ty, tz, gE, gphi, 500)
    assert e.value.code == P.PEPCG_ERR_UNSUPPORTED
    tc.close()


def periodic_problem(n, nt, seed, neutral):
    rng = np.random.default_rng(seed)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0) if neutral else rng.standard_normal(n)
    tx, ty, tz = rng.random(nt), rng.random(nt), rng.random(nt)
    gphi = rng.standard_normal(nt)
    gE = [rng.standard_normal(nt) for _ in range(3)]
    return x, y, z, q, tx, ty, tz, gphi, gE, rng


@pytest.mark.parametrize("corr,neutral", [(0, False), (1, False), (2, False), (2, True)])
def test_periodic_far_field_adjoint_matches_oracle_and_fd(gpu, corr, neutral):
    """27 mirror boxes plus the FMM lattice term, for each extrinsic correction
    (0 none, 1 Redlack, 2 fictitious charges), with the monopole removed
    (random charges) or exactly zero (a neutral box): the GPU adjoint -- walk plus the
    lattice term's transpose -- against the oracle's (whose lattice part
    differentiates the harmonics by dual numbers, not by the ladder relations
    the GPU uses) to 1e-9 of the gradient's scale, and against central FD of
    the GPU forward pass (relative 1e-5, one MAC flip allowed)."""
    x, y, z, q, tx, ty, tz, gphi, gE, rng = periodic_problem(2000, 60, 90 + corr, neutral)
    kw = dict(theta2=0.16, eps2=1e-3, periodicity=(1, 1, 1), fmm_extrinsic_correction=corr)
    grads = {}
    for ff in (0, 1):
        tc = P.TreeCode(precision=P.PRECISION_PLAIN, walk=P.WALK_PER_TARGET,
                        include_far_field_if_periodic=ff, **kw)
        tc.pepc_grow_tree(x, y, z, q)
        if ff:
            assert (tc.last_status == P.PEPCG_WARN_NOT_NEUTRAL) == (not neutral)
        g = tc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
        orc = O.Oracle(walk=0, num_threads=8, include_far_field_if_periodic=ff, **kw)
        if ff:
            orc.set_lattice_coefficients(O.reference_lattice_table(GOLD))
        orc.grow_tree(x, y, z, q)
        go = orc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
        orc.close()
        grads[ff] = (g, go)
        if not ff:
            tc.close()
    g, go = grads[1]
    for k in ("q", "x", "y", "z"):
        scale = np.abs(go[k]).max()
        assert np.abs(g[k] - go[k]).max() <= 1e-9 * scale, k
        # the lattice term's own part (far minus near field), to its own scale
        lat, olat = g[k] - grads[0][0][k], go[k] - grads[0][1][k]
        assert np.abs(olat).max() > 0.0, k
        assert np.abs(lat - olat).max() <= 1e-9 * np.abs(olat).max(), k

    def L(a):
        tc.pepc_grow_tree(a["x"], a["y"], a["z"], a["q"])
        r = tc.pepc_traverse_tree(tx, ty, tz)
        return float(np.sum(gphi * r["pot"] + gE[0] * r["ex"] + gE[1] * r["ey"] + gE[2] * r["ez"]))

    h = 1e-6
    bad = 0
    # a charge perturbed in a neutral box makes it non-neutral and the forward
    # removes the monopole: dL/dq is that (one-sided and FD) derivative
    for trial in range(12):
        j = int(rng.integers(len(x)))
        key = "xyzq"[trial % 4]
        arrs = {"x": x, "y": y, "z": z, "q": q}
        plus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        minus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        plus[key][j] += h
        minus[key][j] -= h
        fd = (L(plus) - L(minus)) / (2 * h)
        an = g[key][j]
        if abs(fd - an) > 1e-5 * max(abs(fd), abs(an), 1e-8):
            bad += 1
    assert bad <= 1, bad
    tc.close()


def test_periodic_far_field_adjoint_mixed_walk(gpu):
    # the benchmark's walk (mixed, 64-target buckets) with the lattice term:
    # its adjoint against the FP64 adjoint of the same bucket walk
    x, y, z, q, tx, ty, tz, gphi, gE, rng = periodic_problem(20000, 2000, 95, True)
    kw = dict(theta2=0.16, eps2=1e-4, walk=P.WALK_GROUP, group_size=64, periodicity=(1, 1, 1))
    out = {}
    for prec in (P.PRECISION_PLAIN, P.PRECISION_MIXED):
        tc = P.TreeCode(precision=prec, **kw)
        tc.pepc_grow_tree(x, y, z, q)
        out[prec] = tc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
        tc.close()
    # without the lattice term the gradient is measurably different
    tn = P.TreeCode(precision=P.PRECISION_PLAIN, include_far_field_if_periodic=0, **kw)
    tn.pepc_grow_tree(x, y, z, q)
    near = tn.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    tn.close()
    for k in ("q", "x", "y", "z"):
        a, b = out[P.PRECISION_MIXED][k], out[P.PRECISION_PLAIN][k]
        rel = np.abs(a - b) / np.abs(b).max()
        assert np.median(rel) < 1e-6, (k, np.median(rel))
        assert np.percentile(rel, 99) < 1e-4, (k, np.percentile(rel, 99))
        # the lattice term is present: the near-field-only gradient differs
        assert np.abs(b - near[k]).max() > 1e-6 * np.abs(b).max(), k


@pytest.mark.parametrize("with_e", [False, True])
def test_adjoint_group64_matches_oracle_buckets(gpu, with_e):
    # the FP64 adjoint of the group walk with 64-target buckets against the
    # oracle's adjoint of the same bucket lists (walk 2, tile_size 64)
    x, y, z, q, tx, ty, tz, gphi, gE, rng = problem(4000, 300, 72)
    if not with_e:
        gE = [np.zeros(len(tx))] * 3
    kw = dict(theta2=0.16, eps2=1e-3)
    tc = P.TreeCode(precision=P.PRECISION_PLAIN, walk=P.WALK_GROUP, group_size=64, **kw)
    tc.pepc_grow_tree(x, y, z, q)
    g = tc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    orc = O.Oracle(walk=2, tile_size=64, **kw)
    orc.grow_tree(x, y, z, q)
    go = orc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    for k in ("q", "x", "y", "z"):
        scale = np.abs(go[k]).max()
        assert np.abs(g[k] - go[k]).max() <= 1e-9 * scale, k
    tc.close()
    orc.close()


@pytest.mark.parametrize("with_e", [False, True])
def test_mixed_adjoint_group64_against_fp64(gpu, with_e):
    # the benchmark's walk (mixed, 64-target buckets): its adjoint on the
    # forward's FP32 lists, in FP32 with FP64 sums across buckets, against the
    # FP64 adjoint of the same bucket walk (the lists differ only where a MAC
    # decision is within FP32 rounding of its threshold)
    x, y, z, q, tx, ty, tz, gphi, gE, rng = problem(20000, 2000, 73)
    if not with_e:
        gE = [np.zeros(len(tx))] * 3
    kw = dict(theta2=0.16, eps2=1e-4, walk=P.WALK_GROUP, group_size=64)
    out = {}
    for prec in (P.PRECISION_PLAIN, P.PRECISION_MIXED):
        tc = P.TreeCode(precision=prec, **kw)
        tc.pepc_grow_tree(x, y, z, q)
        out[prec] = tc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
        tc.close()
    for k in ("q", "x", "y", "z"):
        a, b = out[P.PRECISION_MIXED][k], out[P.PRECISION_PLAIN][k]
        rel = np.abs(a - b) / np.abs(b).max()
        assert np.median(rel) < 1e-6, (k, np.median(rel))
        assert np.percentile(rel, 99) < 1e-4, (k, np.percentile(rel, 99))


def test_mixed_adjoint_configuration_against_direct(gpu):
    # the adjoint configuration through the benchmark's walk (mixed, 64-target
    # buckets) against the FP64 direct-sum gradient
    n, nt = 262144, 4096
    rng = np.random.default_rng(4)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = np.random.default_rng(41).standard_normal(n)
    prng = np.random.default_rng(42)
    tx, ty, tz = (0.25 + 0.5 * prng.random(nt) for _ in range(3))
    q_t = np.random.default_rng(43).standard_normal(n)
    kw = dict(theta2=0.16, eps2=1e-6, walk=P.WALK_GROUP, precision=P.PRECISION_MIXED)
    tt = P.TreeCode(**kw)
    tt.pepc_grow_tree(x, y, z, q_t)
    phi_t = tt.pepc_traverse_tree(tx, ty, tz)["pot"]
    tt.close()
    tc = P.TreeCode(**kw)
    tc.pepc_grow_tree(x, y, z, q)
    phi = tc.pepc_traverse_tree(tx, ty, tz)["pot"]
    gphi = 2.0 * (phi - phi_t)
    zero = [np.zeros(nt)] * 3
    g = tc.traverse_adjoint(tx, ty, tz, zero, gphi, n)
    tc.close()
    orc = O.Oracle(theta2=0.16, eps2=1e-6, walk=0, num_threads=16)
    orc.grow_tree(x, y, z, q)
    gd = orc.traverse_adjoint(tx, ty, tz, zero, gphi, n, direct=True)
    orc.close()
    for k in ("q", "x", "y", "z"):
        rel = np.abs(g[k] - gd[k]) / np.abs(gd[k]).max()
        assert np.median(rel) < 1e-3, (k, np.median(rel))
