"""Test-only kernel set for the Z-slab solver: the oracle's float32 operators applied to padded
CPU slabs, so the solver's host logic (halo planes, walls, level plan, agglomeration, CG over
slabs) runs on the CPU under gloo ranks.  It mirrors ``slab.SlabKernels`` call for call; the
package never imports it."""
import numpy as np
import torch

from oracle import mg as M, tfops

G = 2  # halo planes a side, as slab.GHOST


class OracleSlabKernels:
    def operator(self, kind, level, slab, fields, base):
        sc = base.scale * level.scale
        if kind == "sigma7":
            return M.Sigma7(*(f[slab].numpy() for f in fields), c=base.c, scale=sc)
        if kind == "const7":
            kz, ky, kx = base.k
            return M.const7(kz, ky, kx, sc)
        return M.Stencil27(base.K, sc)

    def jacobi(self, lv, s, src, rhs, dst, omega):
        w = np.zeros(tuple(rhs[s].shape), np.float32) if src is None else src[s].numpy()
        dst[s] = torch.from_numpy(M.jacobi(lv.ops[s], w, rhs[s].numpy(), omega))

    def residual_restrict(self, lv, s, phi, rhs, coarse):
        rc = tfops.restrict_avg(M.residual(lv.ops[s], phi[s].numpy(), rhs[s].numpy()))
        coarse[s, 1:1 + rc.shape[0]] = torch.from_numpy(rc)

    def prolong_correct_smooth(self, lv, s, phi, wc, rhs, dst, omega):
        n = lv.Zp // 2
        c = phi[s].numpy() - tfops.prolong_nearest(wc[s, 1:1 + n].numpy())
        dst[s] = torch.from_numpy(M.jacobi(lv.ops[s], c, rhs[s].numpy(), omega))

    def apply(self, lv, s, src, dst):
        dst[s] = torch.from_numpy(lv.ops[s].apply(src[s].numpy()))

    def residual(self, lv, s, phi, rhs, dst):
        dst[s] = torch.from_numpy(M.residual(lv.ops[s], phi[s].numpy(), rhs[s].numpy()))

    def restrict_interior(self, fine, coarse):
        Zl = fine.shape[1] - 2 * G
        for s in range(fine.shape[0]):
            coarse[s, G:G + Zl // 2] = torch.from_numpy(tfops.restrict_avg(fine[s, G:G + Zl].numpy()))

    def dot(self, x, y, out, scratch):
        Zl = x.shape[1] - 2 * G
        for s in range(x.shape[0]):
            out[s] = (x[s, G:G + Zl].double() * y[s, G:G + Zl].double()).sum()

    def scratch_bytes(self, shape):
        return 8

    def update_xr(self, x, r, p, q, num, den):
        Zl = x.shape[1] - 2 * G
        a = np.float32(float(num.item()) / float(den.item()))
        xi, ri = x[:, G:G + Zl].numpy(), r[:, G:G + Zl].numpy()
        xi[...] = xi + a * p[:, G:G + Zl].numpy()
        ri[...] = ri - a * q[:, G:G + Zl].numpy()

    def update_p(self, p, z, num, den):
        Zl = p.shape[1] - 2 * G
        b = np.float32(0.0)
        if den is not None and float(den.item()) != 0.0:
            b = np.float32(float(num.item()) / float(den.item()))
        pi = p[:, G:G + Zl].numpy()
        zi = z[:, G:G + Zl].numpy()
        pi[...] = zi if b == 0 else zi + b * pi
