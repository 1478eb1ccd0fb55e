"""Seeded synthetic inputs for the anisotropic potential problems.

The reference's own inputs (``mesh_*_sk.npy`` geometries, resistivity data) are not in its
repository, so every workload here is generated from a fixed seed:

* ``anisotropic_sigma``: per axis a field of iid N(0,1) values, smoothed by a 5^3 box
  filter with reflected edges, rescaled to mean 0 and standard deviation ``log_std``, then
  exponentiated (log-normal diagonal conductivity sigma = (sx, sy, sz)).
* ``dipole``: +1 and -1 point sources at two seeded interior cells at least ``margin``
  cells from every wall.
* ``reference_box_source``: the 40^3 unit box at offset 43 that the reference's steady
  solve uses as right-hand side and initial guess
  (``Anisotropic_3d_Multigrid_7point.ipynb`` cell 13), scaled to the grid.
"""
import numpy as np


def _box5(a):
    from scipy.ndimage import uniform_filter
    return uniform_filter(a, size=5, mode="reflect")


def anisotropic_sigma(shape, seed, log_std=1.0, dtype=np.float32):
    """Return sigma as an array ``(3, Z, Y, X)`` ordered (sx, sy, sz)."""
    rng = np.random.default_rng(seed)
    out = np.empty((3,) + tuple(shape), dtype=dtype)
    for k in range(3):
        g = _box5(rng.standard_normal(shape))
        g = (g - g.mean()) / (g.std() + 1e-30) * log_std
        out[k] = np.exp(g)
    return out


def dipole(shape, seed, margin=4, dtype=np.float32):
    rng = np.random.default_rng(seed + 7919)
    f = np.zeros(shape, dtype=dtype)
    lo = [min(margin, (n - 1) // 2) for n in shape]
    hi = [max(n - margin, l + 1) for n, l in zip(shape, lo)]
    p = tuple(int(rng.integers(l, h)) for l, h in zip(lo, hi))
    while True:
        q = tuple(int(rng.integers(l, h)) for l, h in zip(lo, hi))
        if q != p:
            break
    f[p] = 1.0
    f[q] = -1.0
    return f


def reference_box_source(shape, dtype=np.float32):
    """Unit box of edge 40/128 of the grid at offset 43/128 (reference: 40^3 at 43 on 128^3)."""
    f = np.zeros(shape, dtype=dtype)
    sl = tuple(slice(int(round(43 * n / 128)), int(round(43 * n / 128)) + max(1, int(round(40 * n / 128))))
               for n in shape)
    f[sl] = 1.0
    return f


def random_field(shape, seed, dtype=np.float32):
    return np.random.default_rng(seed).standard_normal(shape).astype(dtype)
