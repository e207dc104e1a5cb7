"""Seeded synthetic particle sets shared by the tests."""
import numpy as np


def cube(n, seed, charges="alt"):
    """Uniform unit cube; charges +1/-1 alternating (pepc-mini's rule) or N(0,1)."""
    rng = np.random.default_rng(seed)
    x, y, z = rng.random(n), rng.random(n), rng.random(n)
    if charges == "alt":
        q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)
    else:
        q = rng.standard_normal(n)
    return x, y, z, q


def plummer(n, seed, rmax=20.0):
    """Plummer sphere (a = 1) truncated at rmax, equal charges 1/n."""
    rng = np.random.default_rng(seed)
    r = np.empty(0)
    while r.size < n:
        u = rng.random(2 * n)
        with np.errstate(divide="ignore"):
            rr = 1.0 / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        r = np.concatenate([r, rr[np.isfinite(rr) & (rr <= rmax)]])
    r = r[:n]
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    p = v * r[:, None]
    return p[:, 0].copy(), p[:, 1].copy(), p[:, 2].copy(), np.full(n, 1.0 / n)


def rocksalt(n):
    """Rock-salt (NaCl) lattice: sites (i + 1/2)/n of the unit cube, q = (-1)^(i+j+k)."""
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    x, y, z = ((i + 0.5) / n).ravel(), ((j + 0.5) / n).ravel(), ((k + 0.5) / n).ravel()
    q = ((-1.0) ** (i + j + k)).ravel()
    return x, y, z, q
