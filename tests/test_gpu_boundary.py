"""GPU: options of the drop-in boundary that frontends set through their
namelists, against the oracle.

  * spatial_interaction_cutoff (module_mirror_boxes.f90:52; pepc-mini reads
    it from its namelist, frontends/pepc-mini/module_helper.f90:82-90): a node
    whose offset from the target has any |component| >= the cutoff is skipped.
    The two reference walks count the skipped node's work differently (the
    pthreads walk counts a skipped leaf, module_tree_walk_pthreads.f90:620-622;
    the simple walk counts nothing, module_tree_walk_simple.f90:330,377), and
    both are reproduced bit for bit;
  * the adjoint with the cutoff skips the same interactions (against the
    oracle's adjoint and FD);
  * the scalar lattice entry point pepcg_lattice_force equals the array form."""
import numpy as np
import pytest

import pepc_b200 as P
from oracle import oracle as O
from tests.datasets import cube

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("walk,owalk", [(P.WALK_PER_TARGET, 0), (P.WALK_PER_TILE, 1),
                                        (P.WALK_GROUP, 2)])
@pytest.mark.parametrize("periodic", [False, True])
def test_spatial_cutoff_bit_exact(gpu, walk, owalk, periodic):
    x, y, z, q = cube(12000, 71, charges="normal")
    cut = (0.3, 0.45, 0.2)
    kw = dict(theta2=0.25, eps2=1e-4, spatial_interaction_cutoff=cut)
    if periodic:
        # mirror boxes with a minimum-image style cutoff, as pepc-b sets it
        # (frontends/pepc-b/pepcb.f90:138), near field only
        kw.update(periodicity=(1, 1, 1), include_far_field_if_periodic=0)
    tc = P.TreeCode(walk=walk, **kw)
    orc = O.Oracle(walk=owalk, tile_size=32 if walk == P.WALK_GROUP else 16, num_threads=8, **kw)
    g = tc.pepc_grow_tree(x, y, z, q)
    go = orc.grow_tree(x, y, z, q)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k
    assert tc.stats()["interactions"] == orc.counters()["interactions"]
    # the cutoff removed interactions: the fields differ from the uncut walk
    tc.set_params(spatial_interaction_cutoff=(np.finfo(np.float64).max,) * 3)
    full = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    assert not np.array_equal(full["pot"], r["pot"])
    tc.close()
    orc.close()


def test_spatial_cutoff_refused_where_not_applied(gpu):
    cut = (0.3, 0.3, 0.3)
    with pytest.raises(P.PepcgError) as e:
        P.TreeCode(precision=P.PRECISION_MIXED, walk=P.WALK_GROUP, spatial_interaction_cutoff=cut)
    assert e.value.code == P.PEPCG_ERR_UNSUPPORTED
    with pytest.raises(P.PepcgError) as e:
        P.TreeCode(spatial_interaction_cutoff=(-1.0, 1.0, 1.0))
    assert e.value.code == P.PEPCG_ERR_BAD_ARG


@pytest.mark.parametrize("walk,owalk", [(P.WALK_PER_TARGET, 0), (P.WALK_GROUP, 2)])
@pytest.mark.parametrize("periodic", [False, True])
def test_spatial_cutoff_adjoint(gpu, walk, owalk, periodic):
    # the adjoint skips exactly the interactions the forward skips: against the
    # oracle's adjoint (1e-9 of each component's scale) and FD of the GPU forward
    x, y, z, q = cube(3000, 73, charges="normal")
    rng = np.random.default_rng(74)
    nt = 60
    tx, ty, tz = rng.random(nt), rng.random(nt), rng.random(nt)
    gphi = rng.standard_normal(nt)
    gE = [rng.standard_normal(nt) for _ in range(3)]
    kw = dict(theta2=0.25, eps2=1e-4, spatial_interaction_cutoff=(0.3, 0.45, 0.2))
    if periodic:
        kw.update(periodicity=(1, 1, 1), include_far_field_if_periodic=0)
    tc = P.TreeCode(walk=walk, group_size=32, **kw)
    tc.pepc_grow_tree(x, y, z, q)
    g = tc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    orc = O.Oracle(walk=owalk, tile_size=32, num_threads=8, **kw)
    orc.grow_tree(x, y, z, q)
    go = orc.traverse_adjoint(tx, ty, tz, gE, gphi, len(x))
    orc.close()
    for k in ("q", "x", "y", "z"):
        assert np.abs(g[k] - go[k]).max() <= 1e-9 * np.abs(go[k]).max(), k

    def L(a):
        tc.pepc_grow_tree(a["x"], a["y"], a["z"], a["q"])
        r = tc.pepc_traverse_tree(tx, ty, tz)
        return float(np.sum(gphi * r["pot"] + gE[0] * r["ex"] + gE[1] * r["ey"] + gE[2] * r["ez"]))

    h, bad = 1e-6, 0
    for trial in range(8):
        j = int(rng.integers(len(x)))
        key = "xyzq"[trial % 4]
        arrs = {"x": x, "y": y, "z": z, "q": q}
        plus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        minus = {k: (v.copy() if k == key else v) for k, v in arrs.items()}
        plus[key][j] += h
        minus[key][j] -= h
        fd = (L(plus) - L(minus)) / (2 * h)
        if abs(fd - g[key][j]) > 1e-5 * np.abs(g[key]).max():
            bad += 1  # a perturbation may flip a MAC or cutoff decision
    assert bad <= 1
    tc.close()


def test_lattice_force_scalar_equals_array_form(gpu):
    rng = np.random.default_rng(73)
    n = 1000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    tc = P.TreeCode(theta2=0.16, periodicity=(1, 1, 1))
    tc.pepc_grow_tree(x, y, z, q)
    pts = rng.random((5, 3))
    arr = tc.lattice(pts[:, 0], pts[:, 1], pts[:, 2])
    for i in range(5):
        e, phi = tc.lattice_force(pts[i])
        assert np.array_equal(e, [arr["ex"][i], arr["ey"][i], arr["ez"][i]])
        assert phi == arr["pot"][i]
    tc.close()
