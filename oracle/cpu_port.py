"""Multi-threaded CPU port of the anisotropic multigrid solve (test and CPU-baseline infrastructure only).

The same discrete operators and the same PCG + V(2,2) weighted-Jacobi algorithm as
``oracle.mg`` (whose numpy arithmetic restates the reference's TensorFlow layers), written
with torch CPU tensor operations so that every host core is used, the way TensorFlow's CPU
kernels (Eigen / oneDNN) run the reference's ``Conv3D`` layers.  It is the timed stand-in
for "the reference TF CPU path" (TensorFlow 2.0, ``environment.yml:31``, cannot be installed
here) and is never called by the product.
"""
import os

import numpy as np
import torch


def _faces(s, c, axis):
    """Face coefficients (lo, hi) along `axis` (-1 x, -2 y, -3 z) with wall ghost sigma =
    interior sigma (``Anisotropic Resistivity Tomography/README:14-26``)."""
    lo = s.clone()
    hi = s.clone()
    n = s.shape[axis]
    if n > 1:
        a = s.narrow(axis, 1, n - 1)
        b = s.narrow(axis, 0, n - 1)
        m = 0.5 * (a + b)
        lo.narrow(axis, 1, n - 1).copy_(m)
        hi.narrow(axis, 0, n - 1).copy_(m)
    return c * lo, c * hi


class Sigma7CPU:
    def __init__(self, sx, sy, sz, scale=1.0):
        self.s = (sx, sy, sz)
        self.scale = scale
        self.f = [_faces(sx, scale, -1), _faces(sy, scale, -2), _faces(sz, scale, -3)]
        self.diag = sum(lo + hi for lo, hi in self.f)

    def apply(self, x):
        out = self.diag * x
        (xl, xh), (yl, yh), (zl, zh) = self.f
        out[..., :, :, 1:] -= xl[..., :, :, 1:] * x[..., :, :, :-1]
        out[..., :, :, :-1] -= xh[..., :, :, :-1] * x[..., :, :, 1:]
        out[..., :, 1:, :] -= yl[..., :, 1:, :] * x[..., :, :-1, :]
        out[..., :, :-1, :] -= yh[..., :, :-1, :] * x[..., :, 1:, :]
        out[..., 1:, :, :] -= zl[..., 1:, :, :] * x[..., :-1, :, :]
        out[..., :-1, :, :] -= zh[..., :-1, :, :] * x[..., 1:, :, :]
        return out

    def coarsen(self, cs):
        r = lambda a: torch.nn.functional.avg_pool3d(a[None, None], 2)[0, 0]
        return Sigma7CPU(r(self.s[0]), r(self.s[1]), r(self.s[2]), self.scale * cs)


def _restrict(a):
    return torch.nn.functional.avg_pool3d(a[None, None], 2)[0, 0]


def _prolong(a):
    return a.repeat_interleave(2, 0).repeat_interleave(2, 1).repeat_interleave(2, 2)


def vcycle(ops, l, phi, f, nu=2, omega=2.0 / 3.0, coarse_sweeps=32):
    op = ops[l]
    if l == len(ops) - 1:
        w = torch.zeros_like(f)
        for _ in range(coarse_sweeps):
            w = w + omega * (f - op.apply(w)) / op.diag
        return w
    for _ in range(nu):
        phi = phi + omega * (f - op.apply(phi)) / op.diag
    fc = _restrict(op.apply(phi) - f)
    wc = vcycle(ops, l + 1, torch.zeros_like(fc), fc, nu, omega, coarse_sweeps)
    phi = phi - _prolong(wc)
    for _ in range(nu):
        phi = phi + omega * (f - op.apply(phi)) / op.diag
    return phi


def hierarchy(sig, n_levels, coarse_scale=0.5):
    ops = [Sigma7CPU(*(torch.from_numpy(np.ascontiguousarray(sig[k], np.float32)) for k in range(3)))]
    for _ in range(n_levels - 1):
        ops.append(ops[-1].coarsen(coarse_scale))
    return ops


def pcg_solve(ops, b, tol=1e-6, max_iter=500):
    """Same algorithm as ``oracle.mg.pcg_solve`` with the V(2,2) preconditioner."""
    b = torch.from_numpy(np.ascontiguousarray(b, np.float32))
    x = torch.zeros_like(b)
    r = b.clone()
    nb = float(torch.linalg.vector_norm(b.double()))
    p = torch.zeros_like(b)
    rz_old = None
    it = 0
    for it in range(1, max_iter + 1):
        z = vcycle(ops, 0, torch.zeros_like(r), r)
        rz = float((r.double() * z.double()).sum())
        p = z + (rz / rz_old if rz_old else 0.0) * p
        rz_old = rz
        q = ops[0].apply(p)
        alpha = rz / float((p.double() * q.double()).sum())
        x = x + alpha * p
        r = r - alpha * q
        if float(torch.linalg.vector_norm(r.double())) / nb < tol:
            break
    return x.numpy(), it


def threads():
    n = os.cpu_count() or 1
    torch.set_num_threads(n)
    return n
