"""CPU: the oracle's time-step pieces (push, external field, periodic wrap)
against direct numpy statements of the reference expressions
(frontends/pepc-mini/module_helper.f90:205-222, :321-334;
module_mirror_boxes.f90:177-218)."""
import numpy as np

from oracle import oracle as O


def test_push_and_external_field():
    rng = np.random.default_rng(61)
    n = 1000
    q, m = rng.standard_normal(n), rng.random(n) + 0.5
    e = [rng.standard_normal(n) for _ in range(3)]
    v = [rng.standard_normal(n) for _ in range(3)]
    x = [rng.random(n) for _ in range(3)]
    dt = 1e-3
    v_ref = [vi + dt * q / m * ei for vi, ei in zip(v, e)]
    x_ref = [xi + dt * vi for xi, vi in zip(x, v_ref)]
    O.push_particles(dt, q, m, e, v, x)
    for a, b in zip(v + x, v_ref + x_ref):
        assert np.array_equal(a, b)
    ez, pot = e[2].copy(), rng.standard_normal(n)
    ez_ref, pot_ref = ez + 0.25, pot - x[2] * 0.25
    O.apply_external_field(0.25, x[2], ez, pot)
    assert np.array_equal(ez, ez_ref) and np.array_equal(pot, pot_ref)


def test_wrap_principal_axes():
    rng = np.random.default_rng(62)
    n = 2000
    c = [rng.uniform(-3.0, 4.0, n) for _ in range(3)]
    walls, origin = (2.0, 1.0, 0.5), (0.1, -0.2, 0.0)
    kw = dict(periodicity=(1, 1, 0), t_lattice_1=(2.0, 0.0, 0.0), t_lattice_2=(0.0, 1.0, 0.0),
              t_lattice_3=(0.0, 0.0, 0.5), lattice_origin=origin)
    ref = [np.mod(c[d] - origin[d], walls[d]) + origin[d] if d < 2 else c[d].copy()
           for d in range(3)]
    O.constrain_periodic(*c, **kw)
    for d in range(3):
        assert np.array_equal(c[d], ref[d])
    assert np.all((c[0] >= 0.1) & (c[0] <= 2.1))


def test_wrap_skewed_lattice_lands_in_the_cell():
    rng = np.random.default_rng(63)
    n = 2000
    c = [rng.uniform(-2.0, 3.0, n) for _ in range(3)]
    t1, t2, t3 = (1.0, 0.0, 0.0), (0.5, 1.0, 0.0), (0.0, 0.3, 1.0)
    O.constrain_periodic(*c, periodicity=(1, 1, 1), t_lattice_1=t1, t_lattice_2=t2,
                         t_lattice_3=t3)
    Lm = np.array([t1, t2, t3])
    lc = np.stack(c, axis=1) @ np.linalg.inv(Lm)
    assert np.all(lc > -1e-12) and np.all(lc < 1 + 1e-12)
