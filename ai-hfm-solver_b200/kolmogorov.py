"""Two-dimensional multigrid in the reference's Conv2D form, and the doubly periodic
Kolmogorov-flow stepper that uses it for its pressure solve.

``Multigrid2D`` runs on (slots, Y, X) fields:

* ``sawtooth(values, b)``: one cycle of ``Unstructured Mesh/Multigrid_2D.ipynb`` cell 18 (zero
  padding, the same 3x3 weights on every level, one Jacobi with omega = 1 per level, coarsest
  level 1 x 1);
* ``iterate(p, f)``: one outer iteration ``p -= V(A p - f)`` of a V(nu1, nu2) cycle with the
  inner fields in float32 or bf16 storage (float32 arithmetic) and the outer residual and
  update in float32 (the pressure solve of config 2, "float32 vs bf16 smoother").

``KolmogorovFlow`` advances u, v on a doubly periodic n x n grid of [0, 2 pi)^2 forced by
sin(4 y) in x: two-stage momentum (the update of ``naiver_stokes_3D.py:580-622`` in 2D),
divergence, a few warm-started pressure cycles, mean removal, projection.  Steps are captured
in CUDA graphs and replayed.

The reference has no Kolmogorov-flow code (its ``2D Kolmogorov Flow`` folder is empty), so the
discretisation choices are this package's: central differences, a 5-point Laplacian, and for
the periodic pressure cycle coarse weights scaled by 1/4 per level (the rediscretised
Laplacian at twice the spacing; measured ~0.13 residual reduction per V(2,2) cycle with
omega 0.8, while the Galerkin factor 1/2 of these transfer operators stalls near 0.8).
"""
import ctypes as C
import math
import time

import numpy as np
import torch

from . import _lib as L
from .ops import _stream

_DT = {"f32": (L.F32, torch.float32), "bf16": (L.BF16, torch.bfloat16)}


def _p(t):
    return C.c_void_p(t.data_ptr() if t is not None else 0)


def _w9(w):
    a = np.asarray(w, np.float64).reshape(9)
    return (C.c_float * 9)(*[float(v) for v in a])


def level_shapes(shape, min_edge=4):
    shapes = [tuple(int(v) for v in shape)]
    while min(shapes[-1]) // 2 >= min_edge and min(shapes[-1]) >= 2:
        shapes.append((shapes[-1][0] // 2, shapes[-1][1] // 2))
    return shapes


def laplace5(h):
    """Weights of A = -L, the 5-point Laplacian with spacing h: (4 phi - neighbours) / h^2."""
    w = np.zeros((3, 3))
    w[0, 1] = w[2, 1] = w[1, 0] = w[1, 2] = -1.0
    w[1, 1] = 4.0
    return w / h ** 2


class Multigrid2D:
    def __init__(self, shape, w9, storage="f32", periodic=True, nu_pre=2, nu_post=2, omega=0.8,
                 coarse_scale=0.25, min_edge=4, coarse_sweeps=32, slots=1, device="cuda",
                 fused_coarse=True, fused_pairs=True):
        if storage not in _DT:
            raise ValueError("storage must be f32 or bf16")
        if nu_pre < 1:
            raise ValueError("nu_pre >= 1")
        self.code, self.tdt = _DT[storage]
        self.storage = storage
        self.shapes = level_shapes(shape, min_edge)
        if int(np.prod(self.shapes[-1])) > 4096:
            raise ValueError("coarsest level above 4096 cells: lower min_edge")
        self.L = len(self.shapes)
        self.slots = slots
        self.flags = L.FLAG_PERIODIC if periodic else 0
        self.nu_pre, self.nu_post, self.omega = nu_pre, nu_post, float(omega)
        self.coarse_sweeps = coarse_sweeps
        # pairs of sweeps in one launch (HFM_FLAG_TWO_SWEEPS) when enabled: the first two
        # pre-sweeps from zero, and the correction + sweep with the next post-sweep
        self.fused_pairs = bool(fused_pairs)
        w = np.asarray(w9, np.float64).reshape(3, 3)
        self.ws = [_w9(w * coarse_scale ** l) for l in range(self.L)]
        # levels of at most 4096 cells run as one fused launch (hfm_subcycle2d) when enabled
        self.l_sub = next((l for l, s in enumerate(self.shapes) if s[0] * s[1] <= 4096), self.L)
        self.fused_coarse = bool(fused_coarse) and self.L - self.l_sub <= 8 and all(
            s[0] % 2 == 0 and s[1] % 2 == 0 for s in self.shapes[self.l_sub:-1])
        if self.fused_coarse:
            self.ws_sub = (C.c_float * (9 * (self.L - self.l_sub)))(
                *[v for l in range(self.l_sub, self.L) for v in self.ws[l]])
        mk = lambda s, dt: torch.zeros((slots,) + s, dtype=dt, device=device)
        self.w = [mk(s, self.tdt) for s in self.shapes]
        self.tmp = [mk(s, self.tdt) for s in self.shapes]
        self.rhs = [mk(s, self.tdt) for s in self.shapes]
        self.r32 = mk(self.shapes[0], torch.float32)  # float32 residual (diagnostics, sawtooth)

    # -------------------------------------------------------------------- V-cycle
    def _jacobi(self, l, base, coarse, sign, rhs, out, omega):
        Y, X = self.shapes[l]
        L.call("hfm_jacobi2d", self.code, self.ws[l], _p(base), _p(coarse), float(sign), _p(rhs),
               _p(out), self.slots, Y, X, float(omega), self.flags, _stream())

    def _cycle(self, l):
        """Approximate solution of A w = rhs[l] from w = 0; returns the tensor holding it."""
        Y, X = self.shapes[l]
        if self.fused_coarse and l == self.l_sub:
            L.call("hfm_subcycle2d", self.code, self.ws_sub, _p(self.rhs[l]), _p(self.w[l]),
                   self.slots, Y, X, self.L - l, self.omega, self.nu_pre, self.nu_post,
                   self.coarse_sweeps, self.flags, _stream())
            return self.w[l]
        if l == self.L - 1:
            L.call("hfm_coarse_jacobi2d", self.code, self.ws[l], _p(self.rhs[l]), _p(self.w[l]),
                   self.slots, Y, X, self.omega, self.coarse_sweeps, self.flags, _stream())
            return self.w[l]
        cur, oth = self.w[l], self.tmp[l]
        done = 1
        if self.fused_pairs and self.nu_pre == 2 and Y % 2 == 0 and X % 2 == 0:
            # both pre-sweeps, the residual and the restriction in one launch
            L.call("hfm_pre2_restrict2d", self.code, self.ws[l], _p(self.rhs[l]), _p(oth),
                   _p(self.rhs[l + 1]), self.slots, Y, X, self.omega, self.flags, _stream())
            cur, oth = oth, cur
            return self._up(l, cur, oth)
        if self.fused_pairs and self.nu_pre >= 2:
            L.call("hfm_jacobi2d", self.code, self.ws[l], None, None, 0.0, _p(self.rhs[l]), _p(oth),
                   self.slots, Y, X, self.omega, self.flags | L.FLAG_TWO_SWEEPS, _stream())
            cur, oth = oth, cur
            done = 2
        else:
            self._jacobi(l, None, None, 0.0, self.rhs[l], cur, self.omega)
        for _ in range(self.nu_pre - done):
            self._jacobi(l, cur, None, 0.0, self.rhs[l], oth, self.omega)
            cur, oth = oth, cur
        L.call("hfm_residual_restrict2d", self.code, self.ws[l], _p(cur), _p(self.rhs[l]),
               _p(self.rhs[l + 1]), self.slots, Y, X, self.flags, _stream())
        return self._up(l, cur, oth)

    def _up(self, l, cur, oth):
        """The coarser levels' cycle, then the correction and post-sweeps of level l (its
        iterate in ``cur``); returns the tensor holding level l's result."""
        Y, X = self.shapes[l]
        wc = self._cycle(l + 1)
        # prolongation + correction w -= P w_c fused with the first post-sweep (and the second)
        if self.fused_pairs and self.nu_post >= 2:
            L.call("hfm_jacobi2d", self.code, self.ws[l], _p(cur), _p(wc), -1.0, _p(self.rhs[l]),
                   _p(oth), self.slots, Y, X, self.omega, self.flags | L.FLAG_TWO_SWEEPS, _stream())
            cur, oth = oth, cur
            done = 2
        else:
            self._jacobi(l, cur, wc, -1.0, self.rhs[l], oth, self.omega if self.nu_post else 0.0)
            cur, oth = oth, cur
            done = 1
        for _ in range(self.nu_post - done):
            self._jacobi(l, cur, None, 0.0, self.rhs[l], oth, self.omega)
            cur, oth = oth, cur
        return cur

    def iterate(self, p, f):
        """p -= V(A p - f): float32 p and f of shape (slots, Y, X)."""
        Y, X = self.shapes[0]
        L.call("hfm_outer_residual2d", self.ws[0], _p(p), _p(f), self.code, _p(self.rhs[0]),
               self.slots, Y, X, self.flags, None, None, _stream())
        w = self._cycle(0)
        L.call("hfm_update2d", _p(p), self.code, _p(w), -1.0, self.slots * Y * X, _stream())

    def solve(self, p, f, cycles):
        for _ in range(cycles):
            self.iterate(p, f)
        if self.flags & L.FLAG_PERIODIC:
            Y, X = self.shapes[0]
            L.call("hfm_mean_subtract2d", _p(p), self.slots, Y * X, _stream())

    def rel_residual(self, p, f):
        Y, X = self.shapes[0]
        L.call("hfm_residual2d", L.F32, self.ws[0], _p(p), _p(f), _p(self.r32), self.slots, Y, X,
               self.flags, _stream())
        r = self.r32.double().flatten(1).norm(dim=1)
        return (r / f.double().flatten(1).norm(dim=1).clamp_min(1e-300)).cpu().numpy()

    # -------------------------------------------------------------------- reference cycle
    def sawtooth(self, values, b):
        """One ``Multigrid_2D.ipynb#c18`` cycle: returns the new ``values`` (a new tensor, as
        the reference rebinds ``values``) from float32 ``values`` and ``b``.  Construct with
        periodic=False, coarse_scale=1, min_edge=1, omega=1, storage f32 for the reference
        form."""
        if self.code != L.F32:
            raise ValueError("the reference cycle runs in float32 storage")
        Y, X = self.shapes[0]
        st = _stream()
        r = self.rhs
        L.call("hfm_residual2d", L.F32, self.ws[0], _p(values), _p(b), _p(r[0]), self.slots, Y, X,
               self.flags, st)
        for l in range(1, self.L):
            Yf, Xf = self.shapes[l - 1]
            L.call("hfm_restrict_avg2d", L.F32, _p(r[l - 1]), _p(r[l]), self.slots, Yf, Xf, st)
        last = self.L - 1
        self._jacobi(last, None, None, 0.0, r[last], self.w[last], self.omega)
        for l in range(last - 1, -1, -1):
            self._jacobi(l, None, self.w[l + 1], 1.0, r[l], self.w[l], self.omega)
        # values - w, then one Jacobi against b, in one pass
        out = torch.empty_like(values)
        L.call("hfm_jacobi2d", L.F32, self.ws[0], _p(values), _p(self.w[0]), -1.0, _p(b), _p(out),
               self.slots, Y, X, self.omega, self.flags | L.FLAG_SAME_LEVEL_CORR, st)
        return out


def _perturbation(n, seed, device):
    """Smooth seeded perturbation: a few random Fourier modes of amplitude ~1."""
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    h = 2 * np.pi / n
    a = np.zeros((n, n))
    for _ in range(8):
        ky, kx = rng.integers(1, 7, 2)
        a += rng.normal() * np.sin(kx * x * h + ky * y * h + rng.uniform(0, 2 * np.pi))
    return torch.from_numpy((a / 8.0).astype(np.float32)).to(device)


class KolmogorovFlow:
    """Doubly periodic Kolmogorov flow on [0, 2 pi)^2: forcing famp sin(fk y) in x, viscosity
    nu; starts from the laminar profile u = famp / (nu fk^2) sin(fk y) plus a seeded
    perturbation of relative size ``eps``."""

    def __init__(self, n=512, nu=1.0 / 40.0, dt=1e-3, famp=1.0, fk=4.0, storage="f32",
                 cycles=3, eps=0.05, seed=0, device="cuda"):
        self.n, self.nu, self.dt, self.famp, self.fk = n, nu, dt, famp, fk
        self.h = 2 * math.pi / n
        self.cycles = cycles
        z = lambda: torch.zeros((n, n), dtype=torch.float32, device=device)
        self.u, self.v, self.p, self.f = z(), z(), z(), z()
        self.bu, self.bv, self.u1, self.v1 = z(), z(), z(), z()
        y = torch.arange(n, device=device, dtype=torch.float32)[:, None] * self.h
        amp = famp / (nu * fk * fk)
        self.u.copy_((amp * torch.sin(fk * y)).expand(n, n))
        self.u += eps * amp * _perturbation(n, seed, device)
        self.v += eps * amp * _perturbation(n, seed + 1, device)
        self.mg = Multigrid2D((n, n), laplace5(self.h), storage=storage, periodic=True,
                              device=device)
        self.steps_done = 0
        self._graphs = {}

    def _stage(self, pu, pv, bu, bv, ou, ov, c):
        L.call("hfm_kolmogorov_stage", _p(pu), _p(pv), _p(bu), _p(bv), _p(ou), _p(ov), self.n,
               self.n, float(c), float(self.dt), float(self.nu), float(self.h), float(self.famp),
               float(self.fk), _stream())

    def step(self):
        """One time step (enqueued on the current stream)."""
        n, st = self.n, _stream()
        self._stage(self.u, self.v, self.u, self.v, self.bu, self.bv, 0.5)
        self._stage(self.bu, self.bv, self.u, self.v, self.u1, self.v1, 1.0)
        L.call("hfm_kolmogorov_divergence", _p(self.u1), _p(self.v1), _p(self.f), n, n,
               float(self.h), float(self.dt), st)
        p, f = self.p.view(1, n, n), self.f.view(1, n, n)
        self.mg.solve(p, f, self.cycles)
        L.call("hfm_kolmogorov_project", _p(self.u1), _p(self.v1), _p(self.p), n, n,
               float(self.h), float(self.dt), st)
        self.u, self.u1 = self.u1, self.u
        self.v, self.v1 = self.v1, self.v
        self.steps_done += 1

    def run(self, steps, per_graph=50):
        """Advance ``steps`` steps, ``per_graph`` of them per replay of a captured CUDA graph
        (an even number, so the velocity buffers are back in place after every replay)."""
        if per_graph % 2:
            raise ValueError("per_graph must be even")
        remaining = steps
        g = self._graphs.get(per_graph)
        if g is None and remaining >= per_graph + 2:
            s = torch.cuda.Stream()
            s.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(s):
                self.step()  # two real steps outside the capture (first-use set-up)
                self.step()
            torch.cuda.current_stream().wait_stream(s)
            remaining -= 2
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                for _ in range(per_graph):
                    self.step()  # recorded, not executed
            self.steps_done -= per_graph
            self._graphs[per_graph] = g
        if g is not None:
            while remaining >= per_graph:
                g.replay()
                self.steps_done += per_graph
                remaining -= per_graph
        for _ in range(remaining):
            self.step()

    def diagnostics(self):
        u, v, h = self.u.double(), self.v.double(), self.h
        div = (torch.roll(u, -1, 1) - torch.roll(u, 1, 1) + torch.roll(v, -1, 0) - torch.roll(v, 1, 0)) / (2 * h)
        n = self.n
        res = self.mg.rel_residual(self.p.view(1, n, n), self.f.view(1, n, n))[0]
        return {"step": self.steps_done, "energy": float(0.5 * (u * u + v * v).mean()),
                "max_abs_div": float(div.abs().max()), "max_u": float(u.abs().max()),
                "pressure_rel_resid": float(res)}


def config2_kolmogorov(n=512, steps=5000, storages=("f32", "bf16"), cycles=3, log_every=500,
                       seed=0):
    """The 2D part of the mixed-precision workload: 512^2 Kolmogorov flow, nu = 1/40, forcing
    sin(4 y), 5000 steps, float32 vs bf16 storage in the pressure cycles."""
    out = {}
    for st in storages:
        kf = KolmogorovFlow(n=n, storage=st, cycles=cycles, seed=seed)
        hist = [kf.diagnostics()]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        done = 0
        while done < steps:
            k = min(log_every, steps - done)
            kf.run(k)
            done += k
            torch.cuda.synchronize()
            hist.append(kf.diagnostics())
        dt = time.perf_counter() - t0
        out[st] = {"seconds": dt, "ms_per_step": 1e3 * dt / steps, "history": hist,
                   "finite": bool(torch.isfinite(kf.u).all() and torch.isfinite(kf.v).all())}
    if len(storages) == 2:
        a, b = (out[s]["history"] for s in storages)
        out["energy_rel_diff_max"] = max(abs(x["energy"] - y["energy"]) / max(abs(x["energy"]), 1e-300)
                                         for x, y in zip(a, b))
    return out
