"""Oracle for the two-dimensional path (test and CPU-baseline infrastructure only): the reference's Conv2D
multigrid and the doubly periodic Kolmogorov-flow stepper built on it.

2D multigrid semantics follow ``Unstructured Mesh/Multigrid_2D.ipynb``: the 3x3 operator is a
``Conv2D(1, 3, 'SAME')`` layer (cell 7; cross-correlation, zero padding, kernel ``w2[0][a][b][0]``
multiplying ``phi[y + a - 1][x + b - 1]``), restriction a ``Conv2D(1, 2, strides=2, 'VALID')``
with weights 0.25 (cell 9), prolongation ``UpSampling2D(2)`` (cell 11), and the sawtooth cycle
of cell 18.  ``periodic=True`` wraps around instead of zero padding (the Kolmogorov flow).

The reference has no Kolmogorov-flow code: the stepper restates, in two dimensions, the
two-stage momentum update of ``Anisotropic Resistivity Tomography/scripts/
naiver_stokes_3D.py:580-622`` with central differences and a 5-point Laplacian, and its
projection ``:631-633``; arrays are (Y, X), x fastest.
"""
import numpy as np


def conv2d(x, w9, periodic=False, dt=np.float32):
    """Cross-correlation of (Y, X) with a 3x3 kernel, zero or periodic padding."""
    x = np.asarray(x, dt)
    w = np.asarray(w9, dt).reshape(3, 3)
    xp = np.pad(x, 1, mode="wrap" if periodic else "constant")
    Y, X = x.shape
    out = np.zeros_like(x)
    for a in range(3):
        for b in range(3):
            out += w[a, b] * xp[a:a + Y, b:b + X]
    return out


def restrict2d(x):
    """2x2 VALID average with weight 0.25 (odd extents floored)."""
    x = np.asarray(x)
    Y, X = (x.shape[0] // 2) * 2, (x.shape[1] // 2) * 2
    x = x[:Y, :X]
    s = (x[0::2, 0::2] + x[0::2, 1::2]) + (x[1::2, 0::2] + x[1::2, 1::2])
    return (np.asarray(0.25, x.dtype) * s).astype(x.dtype)


def prolong2d(x):
    return np.repeat(np.repeat(np.asarray(x), 2, axis=0), 2, axis=1)


def jacobi2d(w9, phi, rhs, omega=1.0, periodic=False, dt=np.float32):
    """phi + omega (rhs - A phi) / w[1, 1]."""
    w = np.asarray(w9, dt).reshape(3, 3)
    phi = np.asarray(phi, dt)
    return phi + dt(omega) * (np.asarray(rhs, dt) - conv2d(phi, w, periodic, dt)) / w[1, 1]


def level_shapes(shape, min_edge=1):
    shapes = [tuple(shape)]
    while min(shapes[-1]) // 2 >= min_edge and min(shapes[-1]) >= 2:
        shapes.append((shapes[-1][0] // 2, shapes[-1][1] // 2))
    return shapes


def sawtooth2d(w9, values, b, n_levels, keep=None):
    """One cycle of ``Multigrid_2D.ipynb#c18`` (j_itr = 1): r = A v - b, restriction to the
    coarsest level, w = 0 there, one Jacobi per level on the way up against the restricted
    residual, one on the fine level against r, v -= w, then one Jacobi on v against b.  The
    same weights on every level, zero padding, omega = 1 (the reference's update
    ``w - A(w)/d + r/d``).  ``keep`` (a dict) receives the residuals and corrections per level
    (level 0 finest)."""
    f32 = np.float32
    r = conv2d(values, w9) - np.asarray(b, f32)
    rs = [r]
    for _ in range(n_levels - 1):
        rs.append(restrict2d(rs[-1]))
    w = np.zeros_like(rs[-1])
    w = jacobi2d(w9, w, rs[-1])
    ws = {n_levels - 1: w}
    for lvl in range(n_levels - 2, -1, -1):
        w = jacobi2d(w9, prolong2d(w), rs[lvl])
        ws[lvl] = w
    if keep is not None:
        keep["r"], keep["w"] = rs, ws
    values = np.asarray(values, f32) - w
    return jacobi2d(w9, values, b)


class VCycle2D:
    """V(nu1, nu2) cycle for the correction w of A w = r (r = A p - f), the sequence the GPU
    path runs: pre-smoothing from w = 0, residual + restriction, recursion, prolongation +
    correction (w -= P w_c) fused with the first post-sweep, the remaining post-sweeps; the
    coarsest level runs ``coarse_sweeps`` Jacobi sweeps from zero.  Coarse weights are the fine
    weights times ``coarse_scale`` per level."""

    def __init__(self, w9, shape, periodic=True, nu_pre=2, nu_post=2, omega=0.8,
                 coarse_scale=0.25, min_edge=4, coarse_sweeps=32, dt=np.float64):
        self.shapes = level_shapes(shape, min_edge)
        self.ws = [np.asarray(w9, np.float64).reshape(3, 3) * coarse_scale ** l
                   for l in range(len(self.shapes))]
        self.periodic, self.nu_pre, self.nu_post = periodic, nu_pre, nu_post
        self.omega, self.coarse_sweeps, self.dt = omega, coarse_sweeps, dt

    def _j(self, l, phi, rhs, omega=None):
        return jacobi2d(self.ws[l], phi, rhs, self.omega if omega is None else omega,
                        self.periodic, self.dt)

    def cycle(self, l, rhs):
        dt = self.dt
        if l == len(self.shapes) - 1:
            w = np.zeros(self.shapes[l], dt)
            for _ in range(self.coarse_sweeps):
                w = self._j(l, w, rhs)
            return w
        w = np.zeros(self.shapes[l], dt)
        for _ in range(self.nu_pre):
            w = self._j(l, w, rhs)
        rc = restrict2d(conv2d(w, self.ws[l], self.periodic, dt) - rhs)
        wc = self.cycle(l + 1, rc)
        w = w - prolong2d(wc)
        for _ in range(max(self.nu_post, 1)):
            w = self._j(l, w, rhs, self.omega if self.nu_post else 0.0)
        return w

    def solve(self, p, f, cycles):
        """``cycles`` outer iterations p -= V(A p - f); the mean of p removed at the end
        (periodic)."""
        p = np.asarray(p, self.dt).copy()
        for _ in range(cycles):
            r = conv2d(p, self.ws[0], self.periodic, self.dt) - np.asarray(f, self.dt)
            p = p - self.cycle(0, r)
        if self.periodic:
            p = p - p.mean()
        return p

    def rel_residual(self, p, f):
        r = conv2d(p, self.ws[0], self.periodic, np.float64) - np.asarray(f, np.float64)
        return np.linalg.norm(r) / max(np.linalg.norm(f), 1e-300)


def laplace5(h):
    """Weights of A = -L (5-point): (4 phi - neighbours) / h^2."""
    w = np.zeros((3, 3))
    w[0, 1] = w[2, 1] = w[1, 0] = w[1, 2] = -1.0
    w[1, 1] = 4.0
    return w / h ** 2


def ns_stage(pu, pv, bu, bv, c, dt, nu, h, famp, fk, dtype=np.float32):
    """base + c dt (nu L phi - U dphi/dx - V dphi/dy + F) for both components."""
    t = dtype
    pu, pv = np.asarray(pu, t), np.asarray(pv, t)
    sh = lambda a, dy, dx: np.roll(np.roll(a, -dy, axis=0), -dx, axis=1)  # a[y + dy, x + dx]
    ih2, i2h = t(1.0 / (h * h)), t(0.5 / h)
    lap = lambda a: (sh(a, 0, -1) + sh(a, 0, 1) + sh(a, -1, 0) + sh(a, 1, 0) - t(4) * a) * ih2
    ddx = lambda a: (sh(a, 0, 1) - sh(a, 0, -1)) * i2h
    ddy = lambda a: (sh(a, 1, 0) - sh(a, -1, 0)) * i2h
    Y = pu.shape[0]
    force = (t(famp) * np.sin(t(fk) * np.arange(Y, dtype=t) * t(h)).astype(t))[:, None]
    ou = bu + t(c) * t(dt) * (t(nu) * lap(pu) - pu * ddx(pu) - pv * ddy(pu) + force)
    ov = bv + t(c) * t(dt) * (t(nu) * lap(pv) - pu * ddx(pv) - pv * ddy(pv))
    return ou.astype(t), ov.astype(t)


def ns_divergence(u, v, h, dt):
    i2h = 0.5 / h
    div = (np.roll(u, -1, 1) - np.roll(u, 1, 1)) * i2h + (np.roll(v, -1, 0) - np.roll(v, 1, 0)) * i2h
    return -div / dt


def ns_project(u, v, p, h, dt):
    i2h = 0.5 / h
    return (u - dt * (np.roll(p, -1, 1) - np.roll(p, 1, 1)) * i2h,
            v - dt * (np.roll(p, -1, 0) - np.roll(p, 1, 0)) * i2h)


def ns_step(u, v, p, mg, cycles, dt, nu, h, famp=1.0, fk=4.0):
    """One step: two-stage momentum, divergence, `cycles` pressure cycles from the previous
    p, projection.  Returns (u, v, p)."""
    bu, bv = ns_stage(u, v, u, v, 0.5, dt, nu, h, famp, fk)
    u1, v1 = ns_stage(bu, bv, u, v, 1.0, dt, nu, h, famp, fk)
    f = ns_divergence(u1, v1, h, dt)
    p = mg.solve(p, f, cycles)
    u2, v2 = ns_project(u1, v1, p, h, dt)
    return u2, v2, p
