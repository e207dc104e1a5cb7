"""CPU: the oracle's adjoint walk (orc_traverse_adjoint) and direct-sum
gradient (orc_direct_adjoint) against central finite differences.

The tree adjoint is the exact derivative of the tree-code fields with the
interaction lists held fixed, so FD of the oracle's forward walk agrees with
it to FD accuracy wherever a perturbation flips no MAC decision; the direct
gradient is checked against FD of a numpy direct sum.  With periodic
boundaries and the FMM lattice term (each extrinsic correction) the adjoint
adds the lattice term's transpose, whose harmonic gradients come from dual
numbers; checked against FD of the oracle's full periodic forward pass."""
import numpy as np
import pytest

from oracle import oracle as O


def _problem(n, nt, seed):
    rng = np.random.default_rng(seed)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = rng.standard_normal(n)
    tx, ty, tz = (0.25 + 0.5 * rng.random(nt) for _ in range(3))
    gphi = rng.standard_normal(nt)
    gE = [rng.standard_normal(nt) for _ in range(3)]
    return x, y, z, q, tx, ty, tz, gphi, gE, rng


def _L_tree(arrs, t, gphi, gE, **kw):
    o = O.Oracle(**kw)
    o.grow_tree(arrs["x"], arrs["y"], arrs["z"], arrs["q"])
    r = o.traverse_tree(*t)
    o.close()
    return float(np.sum(gphi * r["pot"] + gE[0] * r["ex"] + gE[1] * r["ey"] + gE[2] * r["ez"]))


def _L_direct(arrs, t, gphi, gE, eps2):
    dx = t[0][:, None] - arrs["x"][None, :]
    dy = t[1][:, None] - arrs["y"][None, :]
    dz = t[2][:, None] - arrs["z"][None, :]
    r2 = dx * dx + dy * dy + dz * dz + eps2
    rinv = 1.0 / np.sqrt(r2)
    r3 = rinv ** 3
    q = arrs["q"][None, :]
    pot = np.sum(q * rinv, axis=1)
    ex, ey, ez = (np.sum(q * d * r3, axis=1) for d in (dx, dy, dz))
    return float(np.sum(gphi * pot + gE[0] * ex + gE[1] * ey + gE[2] * ez))


@pytest.mark.parametrize("direct,walk", [(False, 0), (True, 0), (False, 2)])
def test_oracle_adjoint_against_fd(direct, walk):
    # walk 2: buckets of 64 consecutive targets (the group walk's lists)
    x, y, z, q, tx, ty, tz, gphi, gE, rng = _problem(600, 24 if walk == 0 else 100, 13)
    kw = dict(theta2=0.16, eps2=1e-3, walk=walk, tile_size=64)
    o = O.Oracle(**kw)
    o.grow_tree(x, y, z, q)
    g = o.traverse_adjoint(tx, ty, tz, gE, gphi, len(x), direct=direct)
    o.close()
    t = (tx, ty, tz)
    h = 1e-6
    bad = 0
    for trial in range(24):
        j = int(rng.integers(len(x)))
        key = "xyzq"[trial % 4]
        arrs = {"x": x, "y": y, "z": z, "q": q}
        plus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        minus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        plus[key][j] += h
        minus[key][j] -= h
        if direct:
            fd = (_L_direct(plus, t, gphi, gE, 1e-3) - _L_direct(minus, t, gphi, gE, 1e-3)) / (2 * h)
        else:
            fd = (_L_tree(plus, t, gphi, gE, **kw) - _L_tree(minus, t, gphi, gE, **kw)) / (2 * h)
        an = g[key][j]
        if abs(fd - an) > 1e-5 * max(abs(fd), abs(an), 1e-6):
            bad += 1
    assert bad <= (0 if direct else 1), bad


def test_oracle_adjoint_close_to_direct_gradient():
    x, y, z, q, tx, ty, tz, gphi, gE, _ = _problem(2000, 32, 17)
    o = O.Oracle(theta2=0.16, eps2=1e-3, walk=0)
    o.grow_tree(x, y, z, q)
    gt = o.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    gd = o.traverse_adjoint(tx, ty, tz, gE, gphi, len(x), direct=True)
    o.close()
    for k in ("q", "x", "y", "z"):
        rel = np.abs(gt[k] - gd[k]) / np.abs(gd[k]).max()
        assert np.median(rel) < 1e-3, (k, np.median(rel))


@pytest.mark.parametrize("corr,neutral", [(0, False), (1, False), (2, False), (2, True)])
def test_oracle_periodic_far_field_adjoint_against_fd(corr, neutral):
    # a neutral box keeps omega(0, 0) = 0; perturbing a charge there removes
    # the monopole, and the adjoint gives that (FD) derivative
    rng = np.random.default_rng(3)
    n, nt = 300, 20
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0) if neutral else rng.standard_normal(n)
    tx, ty, tz = (rng.random(nt) for _ in range(3))
    gphi = rng.standard_normal(nt)
    gE = [rng.standard_normal(nt) for _ in range(3)]
    kw = dict(theta2=0.16, eps2=1e-3, periodicity=(1, 1, 1), fmm_extrinsic_correction=corr,
              num_threads=8)
    o = O.Oracle(**kw)
    o.grow_tree(x, y, z, q)
    g = o.traverse_adjoint(tx, ty, tz, gE, gphi, n)
    near = O.Oracle(include_far_field_if_periodic=0, **kw)
    near.grow_tree(x, y, z, q)
    gn = near.traverse_adjoint(tx, ty, tz, gE, gphi, n)
    near.close()

    def L(a):
        o.grow_tree(a["x"], a["y"], a["z"], a["q"])
        r = o.traverse_tree(tx, ty, tz)
        return float(np.sum(gphi * r["pot"] + gE[0] * r["ex"] + gE[1] * r["ey"] + gE[2] * r["ez"]))

    h = 1e-6
    for trial in range(12):
        j = int(rng.integers(n))
        key = "xyzq"[trial % 4]
        arrs = {"x": x, "y": y, "z": z, "q": q}
        plus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        minus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        plus[key][j] += h
        minus[key][j] -= h
        fd = (L(plus) - L(minus)) / (2 * h)
        assert abs(fd - g[key][j]) <= 1e-6 * max(abs(fd), 1e-6), (key, j, fd, g[key][j])
        # the lattice term contributes to this coordinate
        assert g[key][j] != gn[key][j]
    o.close()


@pytest.mark.parametrize("law", [2, 4])
def test_oracle_adjoint_other_force_laws_against_fd(law):
    # force_law 2 (2D Coulomb) and 4 (Lennard-Jones): the oracle's adjoint
    # takes the offset derivative by the complex step through the forward
    # kernels and the 2D charge / moment derivatives as fields of unit moments.
    # The Lennard-Jones fields do not depend on the charges, so their dL/dq
    # comes only through the centres of charge and is small next to L: the
    # tolerance is relative to each gradient component's largest entry.
    x, y, z, q, tx, ty, tz, gphi, gE, rng = _problem(400, 16, 5)
    kw = dict(theta2=0.16, eps2=1e-3, force_law=law, walk=0)
    o = O.Oracle(**kw)
    o.grow_tree(x, y, z, q)
    g = o.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    o.close()
    t = (tx, ty, tz)
    h = 1e-5
    for trial in range(16):
        j = int(rng.integers(len(x)))
        key = "xyzq"[trial % 4]
        arrs = {"x": x, "y": y, "z": z, "q": q}
        plus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        minus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        plus[key][j] += h
        minus[key][j] -= h
        fd = (_L_tree(plus, t, gphi, gE, **kw) - _L_tree(minus, t, gphi, gE, **kw)) / (2 * h)
        scale = np.abs(g[key]).max()
        assert abs(fd - g[key][j]) <= 1e-6 * scale, (law, key, j, fd, g[key][j], scale)


def test_oracle_adjoint_refuses_kelbg():
    x, y, z, q, tx, ty, tz, gphi, gE, _ = _problem(100, 4, 6)
    o = O.Oracle(theta2=0.16, eps2=1e-3, force_law=5, kelbg_invsqrttemp=1.0)
    o.grow_tree(x, y, z, np.where(np.arange(100) % 2 == 0, 1.0, -1.0))
    with pytest.raises(RuntimeError):
        o.traverse_adjoint(tx, ty, tz, gE, gphi, 100)
    o.close()


@pytest.mark.parametrize("walk", [0, 2])
def test_oracle_adjoint_spatial_cutoff_against_fd(walk):
    # spatial_interaction_cutoff: the adjoint skips the interactions the walk
    # skips (module_tree_walk_pthreads.f90:622,639; module_tree_walk_simple.f90:330,377)
    x, y, z, q, tx, ty, tz, gphi, gE, rng = _problem(500, 24, 19)
    kw = dict(theta2=0.16, eps2=1e-3, walk=walk, tile_size=32,
              spatial_interaction_cutoff=(0.25, 0.3, 0.2))
    o = O.Oracle(**kw)
    o.grow_tree(x, y, z, q)
    g = o.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    o.close()
    full = O.Oracle(**{k: v for k, v in kw.items() if k != "spatial_interaction_cutoff"})
    full.grow_tree(x, y, z, q)
    gf = full.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    full.close()
    assert not np.array_equal(g["q"], gf["q"])  # the cutoff removed interactions
    t = (tx, ty, tz)
    h, bad = 1e-6, 0
    for trial in range(16):
        j = int(rng.integers(len(x)))
        key = "xyzq"[trial % 4]
        arrs = {"x": x, "y": y, "z": z, "q": q}
        plus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        minus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        plus[key][j] += h
        minus[key][j] -= h
        fd = (_L_tree(plus, t, gphi, gE, **kw) - _L_tree(minus, t, gphi, gE, **kw)) / (2 * h)
        if abs(fd - g[key][j]) > 1e-6 * np.abs(g[key]).max():
            bad += 1  # a perturbation may flip a MAC or cutoff decision
    assert bad <= 1, bad
