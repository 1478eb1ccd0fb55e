"""Z-slab decomposition of one multigrid solve over several GPUs (one process per GPU).

The reference splits its grid into MPI sub-domains, each padded by one halo cell
(``Anisotropic Resistivity Tomography/scripts/halo_exchange.py:431-499``,
``domain_decomposition_3D``), and after every stencil call copies the sub-domain to the host,
swaps the six faces with ``Isend``/``Irecv`` and copies it back (``structured_halo_update_3D``,
``halo_exchange.py:635-719``).  Its parallel multigrid coarsens every sub-domain down to one
cell on its own (``parallel_naiver_stokes_3D.py:745-823``), so parallel and serial answers
differ.

This module keeps the decomposition, not the mechanics:

* the grid is cut along Z only (the outermost axis of the ``[z][y][x]`` layout), so a halo is
  one contiguous plane that NCCL sends from the field itself over NVLink; nothing is packed
  and nothing goes through the host;
* every slab field is stored as ``(Zl + 2 GHOST, Y, X)`` with GHOST = 2 planes on each side.
  The plane next to the interior holds the neighbour's values; the outer one only keeps the
  2x2x2 restriction and the nearest-neighbour prolongation pair-aligned, so the fused library
  kernels (``hfm_residual_restrict``, ``hfm_prolong_correct_smooth``) run on the padded slab
  unchanged.  Whatever a kernel writes into halo planes is discarded and refreshed by the next
  halo update;
* at the physical walls the halo plane holds zero for iterates (the SAME zero padding) and a
  copy of the wall plane for conductivities (ghost sigma = interior sigma), so every interior
  value equals the one-domain value bit for bit;
* coarse levels are agglomerated: once a level is small (``agglomerate_cells``) or a slab can
  no longer be halved along Z, the restricted residual is all-gathered and the rest of the
  V-cycle runs on the whole coarse grid on every rank.  The answer therefore does not depend
  on the number of slabs (no per-slab coarse solves as in the reference).

Communication goes through a slab group: ``DistSlabs`` (``torch.distributed``: NCCL on GPUs,
gloo in CPU tests; one slab per process) or ``LocalSlabs`` (all slabs in one process: the halo
update is a plane copy).  Stencil work goes through a kernel set; ``SlabKernels`` (libhfm) is
the only one in the package.
"""
import ctypes as C
import math

import torch
import torch.distributed as dist

from . import _lib as L
from .multigrid import SolverConfig
from .ops import Const7, Stencil27

GHOST = 2


def level_shapes(shape, n_levels=0, min_edge=4):
    """Halve while every extent is even and the smallest exceeds ``min_edge`` (the rule of
    ``hfm_mg_create`` without an explicit depth), stopping at ``n_levels`` when given."""
    shapes = [tuple(int(v) for v in shape)]
    while n_levels <= 0 or len(shapes) < n_levels:
        z, y, x = shapes[-1]
        if z % 2 or y % 2 or x % 2 or min(z, y, x) <= min_edge:
            break
        shapes.append((z // 2, y // 2, x // 2))
    return shapes


def _walls(x, wall, low, high):
    """Physical-wall halo planes of the first / last slab in ``x`` (S, Zp, Y, X)."""
    G = GHOST
    Zl = x.shape[1] - 2 * G
    if wall == "zero":
        if low:
            x[0, G - 1].zero_()
        if high:
            x[-1, G + Zl].zero_()
    else:  # "mirror": ghost conductivity = wall-plane conductivity
        if low:
            x[0, G - 1].copy_(x[0, G])
        if high:
            x[-1, G + Zl].copy_(x[-1, G + Zl - 1])


# ------------------------------------------------------------------------------ slab groups
class LocalSlabs:
    """``world`` slabs held by this process (batch dimension of every field)."""

    def __init__(self, world=1):
        if world < 1:
            raise ValueError("world must be >= 1")
        self.world = int(world)
        self.first = 0
        self.count = self.world

    def halo(self, x, wall="zero"):
        G = GHOST
        Zl = x.shape[1] - 2 * G
        if self.count > 1:
            x[1:, G - 1].copy_(x[:-1, G + Zl - 1])
            x[:-1, G + Zl].copy_(x[1:, G])
        _walls(x, wall, True, True)

    def allreduce(self, v):
        return v

    def gather(self, part, full):
        """Interior planes of every slab of ``part`` (S, Zp, Y, X) into the interior of
        ``full`` (1, Z + 2 GHOST, Y, X)."""
        G = GHOST
        Zl = part.shape[1] - 2 * G
        full[0, G:G + self.world * Zl].copy_(part[:, G:G + Zl].reshape(-1, *part.shape[2:]))


class DistSlabs:
    """One slab per rank of a ``torch.distributed`` group, in rank order along Z.  Halo planes
    travel by ``batch_isend_irecv`` (NCCL send/recv into the halo planes themselves); the
    coarse-level gather is one all-gather, the dot products one all-reduce each."""

    def __init__(self, group=None):
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.first = self.rank
        self.count = 1
        self.nccl = dist.get_backend(group) == "nccl"

    def _peer(self, r):
        return dist.get_global_rank(self.group, r) if self.group is not None else r

    def halo(self, x, wall="zero"):
        G = GHOST
        Zl = x.shape[1] - 2 * G
        ops = []
        if self.rank > 0:
            lo = self._peer(self.rank - 1)
            ops += [dist.P2POp(dist.isend, x[0, G], lo, self.group),
                    dist.P2POp(dist.irecv, x[0, G - 1], lo, self.group)]
        if self.rank < self.world - 1:
            hi = self._peer(self.rank + 1)
            ops += [dist.P2POp(dist.isend, x[0, G + Zl - 1], hi, self.group),
                    dist.P2POp(dist.irecv, x[0, G + Zl], hi, self.group)]
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        _walls(x, wall, self.rank == 0, self.rank == self.world - 1)

    def allreduce(self, v):
        dist.all_reduce(v, group=self.group)
        return v

    def gather(self, part, full):
        G = GHOST
        Zl = part.shape[1] - 2 * G
        mine = part[0, G:G + Zl]
        dst = full[0, G:G + self.world * Zl]
        if self.nccl:
            dist.all_gather_into_tensor(dst, mine, group=self.group)
        else:
            parts = [torch.empty_like(mine) for _ in range(self.world)]
            dist.all_gather(parts, mine.contiguous(), group=self.group)
            dst.copy_(torch.cat(parts))


# ---------------------------------------------------------------------------- operators
class SlabSigma7:
    """Per-cell conductivities (sx, sy, sz) of the slabs held here, each (S, Zl, Y, X), with
    ``c = (cz, cy, cx)`` = 1/h^2 and ``scale``: the Z-slab form of ``ops.Sigma7``."""

    def __init__(self, sx, sy, sz, c=(1.0, 1.0, 1.0), scale=1.0):
        self.s = (sx, sy, sz)
        self.c = tuple(float(v) for v in c)
        self.scale = float(scale)


# ------------------------------------------------------------------------------ kernels
class SlabKernels:
    """libhfm kernels on padded slab fields.  Stencil calls run per slab (B = 1): the
    library's batch stride is the unpadded grid, the slab's includes its halo."""

    def __init__(self):
        L.lib()  # raises when the library is missing: there is no fallback

    @staticmethod
    def _p(x):
        return C.c_void_p(x.data_ptr())

    @staticmethod
    def _stream():
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def operator(self, kind, level, slab, fields, base):
        """ctypes operator struct for one slab of one level."""
        if kind == "sigma7":
            sx, sy, sz = fields
            s = L.HfmOperator()
            s.kind, s.coef_dtype, s.scale = L.OP_SIGMA7, L.F32, base.scale * level.scale
            for i, v in enumerate(base.c):
                s.c[i] = v
            for i, a in enumerate((sx[slab], sy[slab], sz[slab])):
                s.coef[i] = a.data_ptr()
            return s
        if kind == "const7":
            return Const7(*base.k, scale=base.scale * level.scale).struct()
        return Stencil27(base.K, scale=base.scale * level.scale).struct()

    def jacobi(self, lv, s, src, rhs, dst, omega):
        flags = L.FLAG_ZERO_GUESS if src is None else 0
        L.call("hfm_op_jacobi", C.byref(lv.ops[s]), C.c_void_p(0) if src is None else self._p(src[s]),
               self._p(rhs[s]), self._p(dst[s]), C.c_void_p(0), 1, lv.Zp, lv.Y, lv.X,
               float(omega), 1, flags, self._stream())

    def residual_restrict(self, lv, s, phi, rhs, coarse):
        # fine plane pairs (0,1), (2,3), ... land on coarse planes 1, 2, ...: the coarse
        # interior starts at GHOST as the fine one does
        plane = coarse.shape[2] * coarse.shape[3]
        L.call("hfm_residual_restrict", C.byref(lv.ops[s]), self._p(phi[s]), self._p(rhs[s]),
               C.c_void_p(0), C.c_void_p(coarse[s].data_ptr() + 4 * plane), 1, lv.Zp, lv.Y,
               lv.X, 0, self._stream())

    def prolong_correct_smooth(self, lv, s, phi, wc, rhs, dst, omega):
        plane = wc.shape[2] * wc.shape[3]
        L.call("hfm_prolong_correct_smooth", C.byref(lv.ops[s]), self._p(phi[s]),
               C.c_void_p(wc[s].data_ptr() + 4 * plane), self._p(rhs[s]), self._p(dst[s]), 1,
               lv.Zp, lv.Y, lv.X, float(omega), 0, self._stream())

    def apply(self, lv, s, src, dst):
        L.call("hfm_op_apply", C.byref(lv.ops[s]), self._p(src[s]), self._p(dst[s]), 1, lv.Zp,
               lv.Y, lv.X, self._stream())

    def residual(self, lv, s, phi, rhs, dst):
        L.call("hfm_op_residual", C.byref(lv.ops[s]), self._p(phi[s]), self._p(rhs[s]),
               self._p(dst[s]), 1, lv.Zp, lv.Y, lv.X, 0, self._stream())

    def restrict_interior(self, fine, coarse):
        """Average 2x2x2 blocks of every slab's interior planes into the coarse interior."""
        G = GHOST
        S, Zp, Y, X = fine.shape
        Zl = Zp - 2 * G
        for s in range(S):
            L.call("hfm_restrict_avg", self._p(fine[s, G:]), self._p(coarse[s, G:]), 1, Zl, Y, X,
                   self._stream())

    def dot(self, x, y, out, scratch):
        """out[s] = sum over the interior of slab s of x * y (float64)."""
        G = GHOST
        S, Zp, Y, X = x.shape
        n = (Zp - 2 * G) * Y * X
        L.call("hfm_dot_f64", self._p(x[:, G]), self._p(y[:, G]), n, S, Zp * Y * X,
               self._p(out), self._p(scratch), self._stream())

    def scratch_bytes(self, shape):
        S, Zp, Y, X = shape
        return int(L.lib().hfm_reduce_scratch_bytes((Zp - 2 * GHOST) * Y * X, S))

    def update_xr(self, x, r, p, q, num, den):
        G = GHOST
        S, Zp, Y, X = x.shape
        n = (Zp - 2 * G) * Y * X
        L.call("hfm_cg_update_xr", self._p(x[:, G]), self._p(r[:, G]), self._p(p[:, G]),
               self._p(q[:, G]), self._p(num), self._p(den), n, S, Zp * Y * X, self._stream())

    def update_p(self, p, z, num, den):
        G = GHOST
        S, Zp, Y, X = p.shape
        n = (Zp - 2 * G) * Y * X
        L.call("hfm_cg_update_p", self._p(p[:, G]), self._p(z[:, G]),
               C.c_void_p(0) if num is None else self._p(num),
               C.c_void_p(0) if den is None else self._p(den), n, S, Zp * Y * X, self._stream())


# ------------------------------------------------------------------------------- solver
class _Level:
    def __init__(self, group, S, Zl, Y, X, scale, device):
        self.group = group
        self.S, self.Zl, self.Y, self.X = S, Zl, Y, X
        self.Zp = Zl + 2 * GHOST
        self.scale = scale
        shp = (S, self.Zp, Y, X)
        self.u = torch.zeros(shp, device=device)
        self.t = torch.zeros(shp, device=device)
        self.f = torch.zeros(shp, device=device)
        self.sigma = None
        self.ops = []

    def other(self, cur):
        return self.t if cur is self.u else self.u


class SlabMultigrid:
    """V(nu_pre, nu_post)-cycle multigrid on a grid of global ``shape`` (Z, Y, X) cut into
    Z-slabs by ``group`` (``LocalSlabs`` or ``DistSlabs``), stationary (``cfg.accel ==
    "none"``) or as the preconditioner of conjugate gradients (``"cg"``).  ``op`` is an
    ``ops.Const7``, an ``ops.Stencil27`` or a ``SlabSigma7`` holding this process's slabs.
    Cycle parameters come from ``SolverConfig`` (``nu_pre``, ``nu_post`` >= 1, ``omega``,
    ``coarse_sweeps``, ``coarse_omega``, ``coarse_scale``, ``n_levels``, ``min_coarse_edge``,
    ``tol``, ``max_cycles``).  Fields passed in and out are the interiors of the slabs held
    here, (S, Zl, Y, X) with Zl = Z / world.  ``graphs`` (default: when every slab is in this
    process on a GPU) replays the CG iteration as one CUDA graph; NCCL ranks run it eagerly."""

    def __init__(self, shape, op, cfg=None, group=None, device=None, agglomerate_cells=32 ** 3,
                 kernels=None, graphs=None):
        self.cfg = cfg or SolverConfig()
        if self.cfg.cycle != "V" or self.cfg.accel not in ("none", "cg"):
            raise ValueError("the slab solver runs V-cycles, stationary or with cg")
        if self.cfg.nu_pre < 1 or self.cfg.nu_post < 1 or self.cfg.coarse_sweeps < 1:
            raise ValueError("nu_pre, nu_post and coarse_sweeps must be >= 1")
        self.group = group or LocalSlabs(1)
        self.k = kernels or SlabKernels()
        self.device = torch.device(device) if device is not None else (
            torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available()
            else torch.device("cpu"))
        W = self.group.world
        shapes = level_shapes(shape, self.cfg.n_levels, self.cfg.min_coarse_edge)
        if shapes[0][0] % W:
            raise ValueError("Z = %d is not divisible by %d slabs" % (shapes[0][0], W))
        # distributed levels: the slab halves along Z down to the next level; the first
        # level that is small or whose slab cannot halve (and all below) is agglomerated
        la = len(shapes)
        for l, (z, y, x) in enumerate(shapes):
            last = l == len(shapes) - 1
            ok = z % W == 0 and (last or (z // W) % 2 == 0)
            if l > 0 and z * y * x <= agglomerate_cells:
                ok = False
            if not ok:
                la = l
                break
        if la == 0:
            raise ValueError("Z / slabs must be even when the grid has coarser levels")
        self.la = la
        self.shapes = shapes
        if isinstance(op, SlabSigma7):
            self.kind = "sigma7"
        elif isinstance(op, Const7):
            self.kind = "const7"
        elif isinstance(op, Stencil27):
            self.kind = "k27"
        else:
            raise TypeError("op must be ops.Const7, ops.Stencil27 or slab.SlabSigma7")
        self.op = op
        solo = LocalSlabs(1)
        self.levels = []
        S = self.group.count
        for l, (z, y, x) in enumerate(shapes):
            sc = float(self.cfg.coarse_scale) ** l
            if l < la:
                self.levels.append(_Level(self.group, S, z // W, y, x, sc, self.device))
            else:
                self.levels.append(_Level(solo, 1, z, y, x, sc, self.device))
        self.bridge_f = self.bridge_w = None
        if la < len(shapes):
            z, y, x = shapes[la]
            self.bridge_f = _Level(self.group, S, z // W, y, x, 1.0, self.device).f
            self.bridge_w = torch.zeros_like(self.bridge_f)
        self._set_operator()
        fine = self.levels[0]
        shp = (S, fine.Zp, fine.Y, fine.X)
        self._x = torch.zeros(shp, device=self.device)
        self._r = torch.zeros(shp, device=self.device)
        self._p = torch.zeros(shp, device=self.device)
        self._q = torch.zeros(shp, device=self.device)
        self._sums = torch.zeros(S, dtype=torch.float64, device=self.device)
        self._scal = torch.zeros(4, dtype=torch.float64, device=self.device)  # rz rz_old pq rr
        self._graph = None
        self.graphs = (isinstance(self.group, LocalSlabs) and self.device.type == "cuda"
                       if graphs is None else bool(graphs))
        self._scratch = torch.zeros(max(8, self.k.scratch_bytes(shp)), dtype=torch.uint8,
                                    device=self.device)

    # ----------------------------------------------------------------- set-up
    def _set_operator(self):
        G = GHOST
        if self.kind == "sigma7":
            prev = None
            for l, lv in enumerate(self.levels):
                lv.sigma = tuple(torch.zeros((lv.S, lv.Zp, lv.Y, lv.X), device=self.device)
                                 for _ in range(3))
                for a in range(3):
                    if l == 0:
                        lv.sigma[a][:, G:G + lv.Zl].copy_(self.op.s[a])
                    elif l < self.la:
                        self.k.restrict_interior(prev.sigma[a], lv.sigma[a])
                    elif l == self.la:
                        part = torch.zeros_like(self.bridge_f)
                        self.k.restrict_interior(prev.sigma[a], part)
                        self.group.gather(part, lv.sigma[a])
                    else:
                        self.k.restrict_interior(prev.sigma[a], lv.sigma[a])
                    lv.group.halo(lv.sigma[a], "mirror")
                prev = lv
        for lv in self.levels:
            lv.ops = [self.k.operator(self.kind, lv, s, lv.sigma, self.op) for s in range(lv.S)]

    # ----------------------------------------------------------------- cycle
    def _smooth(self, lv, cur, rhs, omega):
        dst = lv.other(cur)
        for s in range(lv.S):
            self.k.jacobi(lv, s, cur, rhs, dst, omega)
        lv.group.halo(dst)
        return dst

    def _vcycle(self, l, cur, rhs):
        """One V-cycle on level ``l`` from ``cur`` (padded, halos valid; None = zero) for
        A_l u = rhs.  Returns the padded field holding the result, halos valid."""
        cfg = self.cfg
        lv = self.levels[l]
        if l == len(self.levels) - 1:
            cur = None
            for _ in range(cfg.coarse_sweeps):
                cur = self._smooth(lv, cur, rhs, cfg.coarse_omega)
            return cur
        for _ in range(cfg.nu_pre):
            cur = self._smooth(lv, cur, rhs, cfg.omega)
        nxt = self.levels[l + 1]
        if l + 1 < self.la or l >= self.la:
            for s in range(lv.S):
                self.k.residual_restrict(lv, s, cur, rhs, nxt.f)
            wc = self._vcycle(l + 1, None, nxt.f)
        else:
            # agglomeration: every slab's coarse residual to every rank, the coarse cycle on
            # the whole grid, and this rank's planes (with one halo plane a side) back
            for s in range(lv.S):
                self.k.residual_restrict(lv, s, cur, rhs, self.bridge_f)
            self.group.gather(self.bridge_f, nxt.f)
            full = self._vcycle(l + 1, None, nxt.f)
            G, Zl = GHOST, self.bridge_w.shape[1] - 2 * GHOST
            for s in range(lv.S):
                z0 = (self.group.first + s) * Zl
                self.bridge_w[s, G - 1:G + Zl + 1].copy_(full[0, z0 + G - 1:z0 + G + Zl + 1])
            wc = self.bridge_w
        dst = lv.other(cur)
        for s in range(lv.S):
            self.k.prolong_correct_smooth(lv, s, cur, wc, rhs, dst, cfg.omega)
        lv.group.halo(dst)
        cur = dst
        for _ in range(cfg.nu_post - 1):
            cur = self._smooth(lv, cur, rhs, cfg.omega)
        return cur

    # ----------------------------------------------------------------- public API
    def _load(self, dst, src):
        G = GHOST
        lv = self.levels[0]
        want = (lv.S, lv.Zl, lv.Y, lv.X)
        if tuple(src.shape) != want:
            raise ValueError("expected slabs of shape %s, got %s" % (want, tuple(src.shape)))
        dst[:, G:G + lv.Zl].copy_(src)

    def vcycle(self, phi, b):
        """One V-cycle from ``phi`` (slabs held here; None = zero) for A phi = b; returns the
        new iterate's slabs."""
        G = GHOST
        lv = self.levels[0]
        self._load(self._r, b)
        cur = None
        if phi is not None:
            self._load(self._x, phi)
            lv.group.halo(self._x)
            cur = self._x
        out = self._vcycle(0, cur, self._r)
        return out[:, G:G + lv.Zl].clone()

    def _global_dot(self, x, y, dst):
        """dst (one float64 on the device) = sum over every slab of every rank of x * y."""
        self.k.dot(x, y, self._sums, self._scratch)
        if self._sums.numel() > 1:
            torch.sum(self._sums, dim=0, keepdim=True, out=dst)
        else:
            dst.copy_(self._sums)
        return self.group.allreduce(dst)

    def _cg_iteration(self, first):
        """z = V(0, r); p = z + (rz / rz_old) p; q = A p; x += a p, r -= a q with
        a = rz / (p . q); rr = r . r.  Every scalar stays in device memory."""
        lv = self.levels[0]
        x, r, p, q = self._x, self._r, self._p, self._q
        rz, rz_old, pq, rr = (self._scal[i:i + 1] for i in range(4))
        z = self._vcycle(0, None, r)
        self._global_dot(r, z, rz)
        if first:
            self.k.update_p(p, z, None, None)
        else:
            self.k.update_p(p, z, rz, rz_old)
        rz_old.copy_(rz)
        lv.group.halo(p)
        for s in range(lv.S):
            self.k.apply(lv, s, p, q)
        self._global_dot(p, q, pq)
        self.k.update_xr(x, r, p, q, rz, pq)
        self._global_dot(r, r, rr)

    def solve(self, b, phi0=None):
        """Solve A x = b to ``cfg.tol`` relative residual.  Returns (x slabs, stats) with
        stats = {"iterations", "rel_resid", "converged", "history"}.  With ``graphs`` the
        conjugate-gradient iterations after the first replay one captured CUDA graph (same
        kernels, same results); only the convergence check reads back to the host."""
        G = GHOST
        cfg = self.cfg
        lv = self.levels[0]
        b_pad = torch.zeros_like(self._r)
        self._load(b_pad, b)
        rr = self._scal[3:4]
        nb = math.sqrt(float(self._global_dot(b_pad, b_pad, rr).item()))
        x = self._x
        x.zero_()
        if phi0 is not None:
            self._load(x, phi0)
        lv.group.halo(x)
        if nb == 0.0:
            return x[:, G:G + lv.Zl].clone(), {"iterations": 0, "rel_resid": 0.0,
                                               "converged": True, "history": [0.0]}
        r = self._r
        for s in range(lv.S):
            self.k.residual(lv, s, x, b_pad, r)        # A x - b
        r.neg_()                                       # b - A x
        hist = [math.sqrt(float(self._global_dot(r, r, rr).item())) / nb]
        it = 0
        if cfg.accel == "none":
            cur = x
            while hist[-1] >= cfg.tol and it < cfg.max_cycles:
                cur = self._vcycle(0, cur, b_pad)
                for s in range(lv.S):
                    self.k.residual(lv, s, cur, b_pad, r)
                hist.append(math.sqrt(float(self._global_dot(r, r, rr).item())) / nb)
                it += 1
            if cur is not x:
                x.copy_(cur)
        else:
            while hist[-1] >= cfg.tol and it < cfg.max_cycles:
                if it > 0 and self.graphs:
                    if self._graph is None:
                        g = torch.cuda.CUDAGraph()
                        with torch.cuda.graph(g):
                            self._cg_iteration(False)
                        self._graph = g
                    self._graph.replay()
                else:
                    self._cg_iteration(it == 0)
                hist.append(math.sqrt(float(rr.item())) / nb)
                it += 1
        return x[:, G:G + lv.Zl].clone(), {"iterations": it, "rel_resid": hist[-1],
                                           "converged": hist[-1] < cfg.tol, "history": hist}


def split(full, group):
    """The slabs of a whole (Z, Y, X) field held by this process, (S, Zl, Y, X)."""
    Z = full.shape[-3]
    Zl = Z // group.world
    lo = group.first * Zl
    return full[..., lo:lo + group.count * Zl, :, :].reshape(group.count, Zl, *full.shape[-2:]).clone()
