"""Resistivity tomography: misfit of surface potentials and its gradient with respect to
per-cell log-conductivities (sigma_x, sigma_y, sigma_z), behind ``torch.autograd``.

Forward model: for every source s (a +1 / -1 current dipole) solve A(sigma) u_s = q_s with
the anisotropic SIGMA7 operator, record u at the receivers P (cells on the z = 0 plane).
Misfit: J = 1/2 sum_s |P u_s - d_s|^2.  The adjoint reuses the same multigrid solver because
A is symmetric: A lam_s = P^T (P u_s - d_s), and the fused kernel
``hfm_sigma7_grad_logsigma`` forms dJ / d log sigma from (u_s, lam_s) of all sources.
Forward fields are checkpointed per source (the float64 solution of each source, not the
solver's hierarchies) for the backward pass; ``recompute=True`` keeps nothing and solves the
forward problems again in the backward pass.

The solves use float64 iterative refinement around the float32 V-cycle-preconditioned CG
(``accel="ir"``), so the fields reach a relative residual of 1e-10 and gradients can be
checked against central finite differences.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from .multigrid import Multigrid, SolverConfig
from .ops import Sigma7, _stream


@dataclass
class Survey:
    n: int
    q: torch.Tensor         # (S, n, n, n) float32 source fields (+1 / -1 dipoles)
    receivers: torch.Tensor  # (R,) flat indices of receiver cells on the z = 0 plane


def make_survey(n=96, n_src=32, n_rec=64, seed=0, device="cuda", margin=4):
    rng = np.random.default_rng(seed)
    q = torch.zeros((n_src, n, n, n), device=device)
    lo, hi = margin, n - margin
    for s in range(n_src):
        a = tuple(int(v) for v in rng.integers(lo, hi, 3))
        b = a
        while b == a:
            b = tuple(int(v) for v in rng.integers(lo, hi, 3))
        q[(s,) + a] = 1.0
        q[(s,) + b] = -1.0
    cells = rng.choice(n * n, size=n_rec, replace=False)  # (y, x) on the z = 0 plane
    return Survey(n, q, torch.as_tensor(np.sort(cells), dtype=torch.long, device=device))


def true_sigma(n, seed=0, device="cuda"):
    """Homogeneous sigma = 1 with three seeded ellipsoidal anomalies: two conductive (x10)
    and one resistive (x0.1), the same in sx, sy, sz."""
    rng = np.random.default_rng(seed + 17)
    z, y, x = np.meshgrid(*(np.arange(n) + 0.5,) * 3, indexing="ij")
    s = np.ones((n, n, n), np.float32)
    for factor in (10.0, 10.0, 0.1):
        c = rng.uniform(0.25 * n, 0.75 * n, 3)
        r = rng.uniform(0.08 * n, 0.18 * n, 3)
        inside = ((z - c[0]) / r[0]) ** 2 + ((y - c[1]) / r[1]) ** 2 + ((x - c[2]) / r[2]) ** 2 <= 1
        s[inside] = factor
    return torch.from_numpy(np.stack([s, s, s])).to(device)


class ForwardSolver:
    """A multigrid handle with one slot per source of a group; solves all sources of the
    group together for one conductivity."""

    def __init__(self, n, group, tol=1e-10, storage="f32", max_cycles=2000):
        self.n = n
        self.group = group
        self.cfg = SolverConfig(cycle="V", accel="ir", storage=storage, tol=tol,
                                max_cycles=max_cycles)
        self.mg = Multigrid((n, n, n), L.OP_SIGMA7, self.cfg, slots=group)

    def close(self):
        self.mg.close()

    def solve(self, sigma, rhs):
        """sigma: (3, n, n, n) float32; rhs: (k <= group, n, n, n) float32 or float64.
        Returns the float64 solutions (k, n, n, n)."""
        k = rhs.shape[0]
        op = Sigma7(sigma[0], sigma[1], sigma[2])
        for s in range(k):
            self.mg.set_operator(op, slot=s)
            if rhs.dtype == torch.float64:
                self.mg.load_f64(s, rhs[s].contiguous())
            else:
                self.mg.load(s, rhs[s].contiguous())
        # unused slots stay switched off (a zero right-hand side converges at once)
        for s in range(k, self.group):
            self.mg.load(s, torch.zeros((self.n,) * 3, device=rhs.device))
        while True:
            self.mg.run(8)
            st = self.mg.query()
            if not any(x["active"] for x in st):
                break
        bad = [x for x in st[:k] if x["status"] != 0]
        if bad:
            raise RuntimeError("tomography solve failed: %s" % bad)
        return torch.stack([self.mg.fetch_f64(s) for s in range(k)])


def _groups(S, g):
    return [(i, min(S, i + g)) for i in range(0, S, g)]


def _misfit_fields(sigma, survey, d_obs, solver):
    S = survey.q.shape[0]
    J = 0.0
    us, res = [], []
    for a, b in _groups(S, solver.group):
        u = solver.solve(sigma, survey.q[a:b])
        r = u.view(b - a, -1)[:, survey.receivers] - d_obs[a:b]
        J += 0.5 * float((r * r).sum())
        us.append(u)
        res.append(r)
    return J, us, res


def _accumulate_grad(sigma, survey, solver, us, res, recompute):
    n = survey.n
    S = survey.q.shape[0]
    g = torch.zeros((3, n, n, n), dtype=torch.float64, device=sigma.device)
    sx, sy, sz = (sigma[k].contiguous() for k in range(3))
    for gi, (a, b) in enumerate(_groups(S, solver.group)):
        u = solver.solve(sigma, survey.q[a:b]) if recompute else us[gi]
        rhs = torch.zeros((b - a, n * n * n), dtype=torch.float64, device=sigma.device)
        rhs[:, survey.receivers] = res[gi]
        lam = solver.solve(sigma, rhs.view(b - a, n, n, n))
        L.call("hfm_sigma7_grad_logsigma", C.c_void_p(sx.data_ptr()), C.c_void_p(sy.data_ptr()),
               C.c_void_p(sz.data_ptr()), C.c_void_p(u.data_ptr()), C.c_void_p(lam.data_ptr()),
               b - a, n, n, n, 1.0, 1.0, 1.0, C.c_void_p(g[0].data_ptr()),
               C.c_void_p(g[1].data_ptr()), C.c_void_p(g[2].data_ptr()), 1, _stream())
    return g


class LogSigmaMisfit(torch.autograd.Function):
    """J(log sigma) with a hand-written adjoint backward."""

    @staticmethod
    def forward(ctx, log_sigma, survey, d_obs, solver, recompute=False):
        sigma = torch.exp(log_sigma.detach()).float().contiguous()
        J, us, res = _misfit_fields(sigma, survey, d_obs, solver)
        ctx.survey, ctx.solver, ctx.recompute = survey, solver, recompute
        ctx.sigma = sigma
        ctx.in_dtype = log_sigma.dtype
        ctx.us = None if recompute else us  # per-source float64 checkpoints
        ctx.res = res
        return torch.tensor(J, dtype=torch.float64, device=log_sigma.device)

    @staticmethod
    def backward(ctx, gJ):
        g = _accumulate_grad(ctx.sigma, ctx.survey, ctx.solver, ctx.us, ctx.res, ctx.recompute)
        return (gJ * g).to(ctx.in_dtype), None, None, None, None


def misfit(log_sigma, survey, d_obs, solver, recompute=False):
    return LogSigmaMisfit.apply(log_sigma, survey, d_obs, solver, recompute)


def observe(sigma, survey, solver):
    """Synthetic data d_s = P u_s for the conductivity ``sigma``."""
    S = survey.q.shape[0]
    out = []
    for a, b in _groups(S, solver.group):
        u = solver.solve(sigma, survey.q[a:b])
        out.append(u.view(b - a, -1)[:, survey.receivers])
    return torch.cat(out)


def misfit_value(log_sigma, survey, d_obs, solver):
    sigma = torch.exp(log_sigma).float().contiguous()
    return _misfit_fields(sigma, survey, d_obs, solver)[0]


def config4_check(n=96, n_src=32, n_rec=64, n_fd=20, eps=1e-4, seed=0, group=32):
    """The differentiation workload: misfit at a homogeneous start against data from the
    three-ellipsoid model, adjoint gradient, and central finite differences on ``n_fd``
    random cells.  Returns a dict of timings and agreement figures."""
    import time
    survey = make_survey(n=n, n_src=n_src, n_rec=n_rec, seed=seed)
    solver = ForwardSolver(n, group=group, tol=1e-10)
    try:
        d_obs = observe(true_sigma(n, seed=seed), survey, solver)
        logs = torch.zeros((3, n, n, n), dtype=torch.float64, device="cuda", requires_grad=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        J = misfit(logs, survey, d_obs, solver)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        J.backward()
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        g = logs.grad.cpu().numpy()
        rng = np.random.default_rng(seed + 1)
        base = logs.detach()
        errs = []
        for _ in range(n_fd):
            k, z, y, x = (int(rng.integers(0, 3)),) + tuple(int(v) for v in rng.integers(0, n, 3))
            lp, lm = base.clone(), base.clone()
            lp[k, z, y, x] += eps
            lm[k, z, y, x] -= eps
            fd = (misfit_value(lp, survey, d_obs, solver) - misfit_value(lm, survey, d_obs, solver)) / (2 * eps)
            errs.append(abs(fd - g[k, z, y, x]) / max(abs(g).max(), 1e-300))
        return {"n": n, "sources": n_src, "receivers": n_rec, "J": float(J.detach()),
                "grad_max": float(np.abs(g).max()), "forward_s": t1 - t0, "backward_s": t2 - t1,
                "fd_cells": n_fd, "fd_max_err_rel_to_gmax": float(max(errs)),
                "fd_median_err_rel_to_gmax": float(np.median(errs))}
    finally:
        solver.close()
