"""GPU: the five benchmark configurations of this tree code, each at its exact
parameters, against the oracle (a CPU restatement of the reference path) and
the FP64 direct sum.

  C1  N = 32,768 uniform in the unit cube (seed 1), charges +1/-1 alternating,
      eps 0.01, theta 0.6, Hilbert keys (and a Morton run): keys, order and the
      fields of both reference walks bit-identical to the oracle on all targets.
  C2  Coulomb explosion, N = 1,048,576 uniform in the unit sphere (seed 2),
      q = m = 1/N, eps 1e-3, theta 0.3, 10 kick-drift steps (dt 1e-3) on the
      device: the plain walk bit-identical to the oracle on 4,096 sampled
      targets (seed 22) at the first and the last step, the mixed walk within
      1e-4 median of the FP64 direct sum there, and the two trajectories agree.
  C3  the 4M Plummer sphere at theta 0.2 and 0.6 (0.4 is in test_gpu_fullsize):
      see test_gpu_fullsize.py, parametrised over the sweep.
  C4  the adjoint configuration: see test_gpu_adjoint.py.
  C5  rock-salt lattice n = 64 (262,144 ions), periodic, 27 boxes + the FMM
      lattice term, eps 0, theta 0.3: fields against the oracle (near field
      bit-identical, lattice term to 1e-11 of the field scale) on sampled
      targets, and the Madelung estimate; then n = 80 perturbed by N(0, 1e-3)
      (seed 5): plain against the oracle, mixed against the periodic direct
      sum."""
import os

import numpy as np
import pytest
import torch

import pepc_b200 as P
from bench import uniform_sphere
from oracle import oracle as O
from tests.datasets import rocksalt

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.npz"))
MADELUNG = 1.7475645946331822


def config1():
    rng = np.random.default_rng(1)
    p = rng.random((32768, 3))
    q = np.where(np.arange(32768) % 2 == 0, 1.0, -1.0)
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), q


@pytest.mark.parametrize("walk,curve", [(P.WALK_PER_TARGET, P.CURVE_HILBERT),
                                        (P.WALK_PER_TILE, P.CURVE_HILBERT),
                                        (P.WALK_PER_TARGET, P.CURVE_MORTON)])
def test_c1_uniform_32k_bit_exact(gpu, walk, curve):
    x, y, z, q = config1()
    kw = dict(theta2=0.36, eps2=1e-4, curve=curve)
    tc = P.TreeCode(walk=walk, **kw)
    orc = O.Oracle(walk=0 if walk == P.WALK_PER_TARGET else 1, num_threads=8, **kw)
    g = tc.pepc_grow_tree(x, y, z, q)
    go = orc.grow_tree(x, y, z, q)
    assert np.array_equal(g.key, go["key"])
    assert np.array_equal(g.perm, go["perm"])
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k
    tc.close()
    orc.close()


def rel_force_err(E, Ed):
    return np.linalg.norm(E - Ed, axis=0) / np.linalg.norm(Ed, axis=0)


def test_c2_explosion_ten_steps(gpu):
    n = 1048576
    x0, y0, z0 = uniform_sphere(n)
    dt, nsteps = 1e-3, 10
    dev = torch.device("cuda", 0)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    idx = np.sort(np.random.default_rng(22).choice(n, 4096, replace=False))
    kw = dict(theta2=0.09, eps2=1e-6)
    radius = {}
    r0 = float(np.mean(np.sqrt(x0 ** 2 + y0 ** 2 + z0 ** 2)))
    for name, prec, walk in (("mixed", P.PRECISION_MIXED, P.WALK_GROUP),
                             ("plain", P.PRECISION_PLAIN, P.WALK_PER_TARGET)):
        q = torch.full((n,), 1.0 / n, dtype=torch.float64, device=dev)
        zeros = lambda: torch.zeros(n, dtype=torch.float64, device=dev)  # noqa: E731
        st = dict(x=T(x0), y=T(y0), z=T(z0), q=q, m=q.clone(), vx=zeros(), vy=zeros(), vz=zeros())
        tc = P.TreeCode(precision=prec, walk=walk, **kw)
        # the library's device calls are ordered on its stream: put it on
        # torch's, so the torch reads and fills here are ordered with them
        tc.set_stream(torch.cuda.current_stream().cuda_stream)
        key = torch.empty(n, dtype=torch.int64, device=dev)
        perm = torch.empty(n, dtype=torch.int64, device=dev)
        out = [zeros() for _ in range(5)]
        for k in range(nsteps):
            tc.grow_tree_device(st["x"], st["y"], st["z"], st["q"])
            nx, ny, nz, nq, nm, nvx, nvy, nvz = (torch.empty_like(q) for _ in range(8))
            tc.particles_device(key, perm, nx, ny, nz, nq)
            for s_, d_ in ((st["m"], nm), (st["vx"], nvx), (st["vy"], nvy), (st["vz"], nvz)):
                tc.gather_device(s_, d_)
            for o in out:
                o.zero_()
            tc.traverse_self_device(*out)
            if k in (0, nsteps - 1):
                E = torch.stack(out[:3]).cpu().numpy()[:, idx]
                if name == "plain":
                    # the oracle grows the same (key-ordered) particles and walks the samples
                    px, py, pz, pq = (a.cpu().numpy() for a in (nx, ny, nz, nq))
                    orc = O.Oracle(walk=0, num_threads=16, **kw)
                    go = orc.grow_tree(px, py, pz, pq)
                    assert np.array_equal(go["perm"], np.arange(n))  # already in key order
                    ro = orc.traverse_tree(px[idx], py[idx], pz[idx])
                    for j, c in enumerate(("ex", "ey", "ez")):
                        assert np.array_equal(E[j], ro[c]), (k, c)
                    assert np.array_equal(out[3].cpu().numpy()[idx], ro["pot"])
                    orc.close()
                else:
                    d = tc.direct(idx)
                    rel = rel_force_err(E, np.stack([d["ex"], d["ey"], d["ez"]]))
                    assert np.median(rel) <= 1e-4, (k, np.median(rel))
            tc.push_particles_device(dt, nq, nm, out[:3], (nvx, nvy, nvz), (nx, ny, nz))
            st.update(x=nx, y=ny, z=nz, q=nq, m=nm, vx=nvx, vy=nvy, vz=nvz)
        radius[name] = float(torch.sqrt(st["x"] ** 2 + st["y"] ** 2 + st["z"] ** 2).mean())
        tc.close()
    assert abs(radius["mixed"] - radius["plain"]) <= 1e-9 * radius["plain"]
    assert radius["plain"] > r0  # the sphere expands


def periodic_pair(theta2, **kw):
    per = (1, 1, 1)
    tc = P.TreeCode(theta2=theta2, eps2=0.0, periodicity=per, **kw)
    okw = {k: v for k, v in kw.items() if k in ("walk", "include_far_field_if_periodic")}
    orc = O.Oracle(theta2=theta2, eps2=0.0, periodicity=per, num_threads=16, **okw)
    orc.set_lattice_coefficients(O.reference_lattice_table(GOLD))
    return tc, orc


def test_c5_rocksalt_64_madelung(gpu):
    n = 64
    x, y, z, q = rocksalt(n)
    tc, orc = periodic_pair(0.09, walk=P.WALK_PER_TARGET)
    g = tc.pepc_grow_tree(x, y, z, q)
    go = orc.grow_tree(x, y, z, q)
    assert np.array_equal(g.key, go["key"]) and np.array_equal(g.perm, go["perm"])
    r = tc.pepc_traverse_tree(g.x, g.y, g.z)
    m_est = -np.mean(q[g.perm] * r["pot"]) / n
    print(f"Madelung estimate, n = 64, theta = 0.3: {m_est:.6f} (NaCl: 1.747565)")
    assert abs(m_est - MADELUNG) < 5e-3
    idx = np.sort(np.random.default_rng(64).choice(n ** 3, 4096, replace=False))
    ro = orc.traverse_tree(go["x"][idx], go["y"][idx], go["z"][idx])
    assert np.array_equal(r["work"][idx], ro["work"])
    for k in ("ex", "ey", "ez", "pot"):
        scale = np.abs(ro[k]).max()
        assert np.abs(r[k][idx] - ro[k]).max() <= 1e-11 * scale, k
    # the 27-box near field alone is bit-identical
    tn = P.TreeCode(theta2=0.09, eps2=0.0, periodicity=(1, 1, 1), include_far_field_if_periodic=0)
    on = O.Oracle(theta2=0.09, eps2=0.0, periodicity=(1, 1, 1), include_far_field_if_periodic=0,
                  num_threads=16)
    gn = tn.pepc_grow_tree(x, y, z, q)
    gon = on.grow_tree(x, y, z, q)
    rn = tn.pepc_traverse_tree(gn.x[idx], gn.y[idx], gn.z[idx])
    ron = on.traverse_tree(gon["x"][idx], gon["y"][idx], gon["z"][idx])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(rn[k], ron[k]), k
    for t in (tc, tn):
        t.close()
    for o in (orc, on):
        o.close()


def test_c5_rocksalt_80_perturbed_plain_and_mixed(gpu):
    n = 80
    x, y, z, q = rocksalt(n)
    rng = np.random.default_rng(5)
    x, y, z = ((a + rng.normal(0.0, 1e-3, a.size)) % 1.0 for a in (x, y, z))
    N = x.size
    idx = np.sort(np.random.default_rng(55).choice(N, 2048, replace=False))
    tc, orc = periodic_pair(0.09, walk=P.WALK_PER_TARGET)
    g = tc.pepc_grow_tree(x, y, z, q)
    go = orc.grow_tree(x, y, z, q)
    assert np.array_equal(g.perm, go["perm"])
    r = tc.pepc_traverse_tree(g.x, g.y, g.z)
    ro = orc.traverse_tree(go["x"][idx], go["y"][idx], go["z"][idx])
    assert np.array_equal(r["work"][idx], ro["work"])
    for k in ("ex", "ey", "ez", "pot"):
        scale = np.abs(ro[k]).max()
        assert np.abs(r[k][idx] - ro[k]).max() <= 1e-11 * scale, k
    d = tc.direct(idx)
    Ed = np.stack([d["ex"], d["ey"], d["ez"]])
    err_plain = np.median(rel_force_err(np.stack([r["ex"], r["ey"], r["ez"]])[:, idx], Ed))
    tm = P.TreeCode(theta2=0.09, eps2=0.0, periodicity=(1, 1, 1), precision=P.PRECISION_MIXED,
                    walk=P.WALK_GROUP)
    gm = tm.pepc_grow_tree(x, y, z, q)
    rm = tm.pepc_traverse_tree(gm.x, gm.y, gm.z)
    err_mixed = np.median(rel_force_err(np.stack([rm["ex"], rm["ey"], rm["ez"]])[:, idx], Ed))
    # on a near-perfect lattice the field is a small residue of cancelling
    # terms: both forms' relative errors are large, the mixed group walk's
    # (64-target buckets, opened more often) the smaller
    assert err_mixed <= err_plain, (err_mixed, err_plain)
    for t in (tc, tm):
        t.close()
    orc.close()
