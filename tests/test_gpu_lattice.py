"""GPU: the periodic far-lattice term (module_fmm_framework.f90) and the
27-box near field against the oracle, which uses the reference's own
pretabulated unit-cube coefficients; the Madelung constant of NaCl as a
physical known answer.

Tolerance: the lattice term goes through pow/sin/cos/atan2 (CUDA's versus
glibc's last-bit differences), so the comparison is relative 1e-11 of the
field scale rather than bit equality; the near-field walk itself is exact."""
import os

import numpy as np
import pytest

import pepc_b200 as P
from oracle import oracle as O
from tests.datasets import rocksalt

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.npz"))


def pair(theta2, per=(1, 1, 1), **kw):
    tc = P.TreeCode(theta2=theta2, eps2=0.0, periodicity=per, **kw)
    okw = {k: v for k, v in kw.items() if k.startswith("t_lattice") or k == "lattice_origin"}
    orc = O.Oracle(theta2=theta2, eps2=0.0, periodicity=per, num_threads=8, **okw)
    if all(per) and not okw:
        orc.set_lattice_coefficients(O.reference_lattice_table(GOLD))
    return tc, orc


def test_lattice_term_matches_oracle(gpu):
    rng = np.random.default_rng(51)
    n = 3000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    tc, orc = pair(0.16)
    tc.pepc_grow_tree(x, y, z, q)
    orc.grow_tree(x, y, z, q)
    px, py, pz = rng.random(500), rng.random(500), rng.random(500)
    a, b = tc.lattice(px, py, pz), orc.lattice(px, py, pz)
    for k in ("ex", "ey", "ez", "pot"):
        scale = np.abs(b[k]).max()
        assert np.abs(a[k] - b[k]).max() <= 1e-11 * scale, k


@pytest.mark.parametrize("corr", [0, 1, 2])
def test_lattice_term_each_correction_dipolar_box(gpu, corr):
    # random charges: a non-neutral box (monopole removed) with a dipole.
    # With the fictitious charges (2) the dipole is cancelled; without (0) or
    # with the Redlack terms (1) it couples to MLattice(1, m), which the
    # reference's unit-cube table holds at zero
    rng = np.random.default_rng(53 + corr)
    n = 3000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = rng.standard_normal(n)
    tc = P.TreeCode(theta2=0.16, eps2=0.0, periodicity=(1, 1, 1), fmm_extrinsic_correction=corr)
    orc = O.Oracle(theta2=0.16, eps2=0.0, periodicity=(1, 1, 1), fmm_extrinsic_correction=corr,
                   num_threads=8)
    orc.set_lattice_coefficients(O.reference_lattice_table(GOLD))
    tc.pepc_grow_tree(x, y, z, q)
    assert tc.last_status == P.PEPCG_WARN_NOT_NEUTRAL
    orc.grow_tree(x, y, z, q)
    px, py, pz = rng.random(500), rng.random(500), rng.random(500)
    a, b = tc.lattice(px, py, pz), orc.lattice(px, py, pz)
    for k in ("ex", "ey", "ez", "pot"):
        scale = np.abs(b[k]).max()
        assert np.abs(a[k] - b[k]).max() <= 1e-11 * scale, k
    tc.close()
    orc.close()


def test_periodic_traverse_matches_oracle(gpu):
    rng = np.random.default_rng(52)
    x, y, z, q = rocksalt(10)
    x = (x + rng.normal(0, 1e-3, x.size)) % 1.0
    y = (y + rng.normal(0, 1e-3, y.size)) % 1.0
    z = (z + rng.normal(0, 1e-3, z.size)) % 1.0
    tc, orc = pair(0.09)
    g = tc.pepc_grow_tree(x, y, z, q)
    go = orc.grow_tree(x, y, z, q)
    assert np.array_equal(g.key, go["key"])
    r = tc.pepc_traverse_tree(g.x, g.y, g.z)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"])
    assert np.array_equal(r["work"], ro["work"])  # 27 boxes, identical interaction lists
    for k in ("ex", "ey", "ez", "pot"):
        scale = np.abs(ro[k]).max()
        assert np.abs(r[k] - ro[k]).max() <= 1e-11 * scale, k


def test_madelung_constant(gpu):
    n = 16
    x, y, z, q = rocksalt(n)
    tc = P.TreeCode(theta2=0.0, eps2=0.0, periodicity=(1, 1, 1), walk=P.WALK_PER_TARGET)
    g = tc.pepc_grow_tree(x, y, z, q)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z)
    qs = q[g.perm]
    m_est = -np.mean(qs * r["pot"]) / n
    assert abs(m_est - 1.7475645946331822) < 1e-8


def test_noncubic_lattice_matches_oracle(gpu):
    # a 2 x 1 x 1 box: lattice coefficients by the iteration at Lmax_multipole = 20
    rng = np.random.default_rng(53)
    n = 2000
    x, y, z = 2.0 * rng.random(n), rng.random(n), rng.random(n)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    tc, orc = pair(0.16, t_lattice_1=(2.0, 0.0, 0.0))
    g = tc.pepc_grow_tree(x, y, z, q)
    go = orc.grow_tree(x, y, z, q)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"])
    for k in ("ex", "ey", "ez", "pot"):
        scale = np.abs(ro[k]).max()
        assert np.abs(r[k] - ro[k]).max() <= 1e-10 * scale, k


def test_not_neutral_is_a_warning(gpu):
    rng = np.random.default_rng(54)
    n = 500
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    tc = P.TreeCode(theta2=0.16, periodicity=(1, 1, 1))
    tc.pepc_grow_tree(x, y, z, np.ones(n))
    assert tc.last_status == P.PEPCG_WARN_NOT_NEUTRAL
    r = tc.pepc_traverse_tree(x, y, z)
    assert np.all(np.isfinite(r["pot"]))


@pytest.mark.parametrize("walk", [P.WALK_PER_TARGET, P.WALK_PER_TILE])
def test_periodic_near_field_bit_exact(gpu, walk):
    """The 27-box near field alone (no lattice term) is the walk's arithmetic
    only, so both plain walks must equal the oracle bit for bit; the per-tile
    walk packs its 16-target tiles into shared warps."""
    rng = np.random.default_rng(53)
    n = 4000
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    q = rng.standard_normal(n)
    kw = dict(theta2=0.25, eps2=1e-4, periodicity=(1, 1, 1), include_far_field_if_periodic=0)
    tc = P.TreeCode(walk=walk, **kw)
    orc = O.Oracle(walk=0 if walk == P.WALK_PER_TARGET else 1, num_threads=8, **kw)
    g = tc.pepc_grow_tree(x, y, z, q)
    go = orc.grow_tree(x, y, z, q)
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)
    ro = orc.traverse_tree(go["x"], go["y"], go["z"], keys=go["key"])
    for k in ("ex", "ey", "ez", "pot", "work"):
        assert np.array_equal(r[k], ro[k]), k
    assert tc.stats()["interactions"] == orc.counters()["interactions"]
