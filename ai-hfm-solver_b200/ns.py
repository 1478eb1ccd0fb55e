"""Incompressible NS time stepper on the GPU, with the reference's operator surface.

Functions named after the reference (``scripts/naiver_stokes_3D.py`` / ``Urban Modelling/
AI_HFM_v3.ipynb``) operate on (Z, Y, X) float32 CUDA tensors through ``libhfm``:
``boundary_condition_velocity``, ``boundary_condition_pressure``,
``boundary_condition_source`` (folded into ``divergence``), ``bluff_body``, the two-stage
``momentum`` update, ``pressure_gradient`` and ``divergence``.  ``NSStepper`` runs the
reference's step (naiver_stokes_3D.py:571-727): BCs, momentum, immersed body, pressure
gradient, divergence source, multigrid pressure solve, correction.

Pressure solve: ``pressure="reference"`` runs the reference's sawtooth cycle (27-point w5,
coarsest 2^3, no fine-level Jacobi on w, residual and pressure zeroed on x = X-1,
``multi_itr`` cycles); ``pressure="fcycle"`` runs F(2,2) cycles on the same operator to a
relative residual ``p_tol`` each step.
"""
import ctypes as C
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from . import weights as W
from .multigrid import Multigrid, SolverConfig
from .ops import Stencil27, _stream


def _p(t):
    return C.c_void_p(t.data_ptr())


def _w(K):
    a = np.ascontiguousarray(np.asarray(K, np.float32).reshape(27))
    return a, a.ctypes.data_as(C.c_void_p)


def _shape(t):
    Z, Y, X = t.shape
    return Z, Y, X


class _Scratch:
    cache = {}

    @classmethod
    def get(cls, shape, device):
        key = (shape, str(device))
        if key not in cls.cache:
            nb = L.lib().hfm_ns_bc_scratch_bytes(*shape)
            cls.cache[key] = torch.empty(max(nb, 16), dtype=torch.uint8, device=device)
        return cls.cache[key]

    @classmethod
    def get_bytes(cls, nbytes, device):
        key = ("bytes", int(nbytes), str(device))
        if key not in cls.cache:
            cls.cache[key] = torch.empty(max(int(nbytes), 16), dtype=torch.uint8, device=device)
        return cls.cache[key]


def boundary_condition_velocity(u, v, w, ub):
    """In place (naiver_stokes_3D.py:420-447)."""
    Z, Y, X = _shape(u)
    L.call("hfm_ns_bc_velocity", _p(u), _p(v), _p(w), Z, Y, X, float(ub),
           _p(_Scratch.get((Z, Y, X), u.device)), _stream())
    return u, v, w


def boundary_condition_pressure(p):
    """In place (naiver_stokes_3D.py:452-462)."""
    Z, Y, X = _shape(p)
    L.call("hfm_ns_bc_pressure", _p(p), Z, Y, X, _p(_Scratch.get((Z, Y, X), p.device)), _stream())
    return p


def bluff_body(u, v, w, sigma, dt):
    """In place u, v, w /= (1 + dt sigma) (naiver_stokes_3D.py:478-483)."""
    Z, Y, X = _shape(u)
    L.call("hfm_ns_immersed_body", _p(u), _p(v), _p(w), _p(sigma), Z, Y, X, float(dt), _stream())
    return u, v, w


def momentum_stage(adv, base, out, Kdif, Kx, Ky, Kz, coef):
    Z, Y, X = _shape(adv[0])
    keep = [_w(K) for K in (Kdif, Kx, Ky, Kz)]
    L.call("hfm_ns_momentum", *(_p(t) for t in adv), *(_p(t) for t in base), *(_p(t) for t in out),
           Z, Y, X, *(k[1] for k in keep), float(coef), _stream())
    return out


def momentum_stage_pg(adv, base, out, k, Kx, Ky, Kz, coef):
    """out = base + coef (k - adv . grad adv_f): the stage of INHALE_demo.ipynb cell 24 with
    the Petrov-Galerkin terms k = (k_x, k_y, k_z) in place of the diffusion stencil."""
    Z, Y, X = _shape(adv[0])
    keep = [_w(K) for K in (Kx, Ky, Kz)]
    L.call("hfm_ns_momentum_pg", *(_p(t) for t in adv), *(_p(t) for t in base),
           *(_p(t) for t in out), *(_p(t) for t in k), Z, Y, X, *(kk[1] for kk in keep),
           float(coef), _stream())
    return out


def pg_dissipation(u, v, w, sigma, out, Kdif, Kx, Ky, Kz, dt, eps_k=1e-3):
    """Petrov-Galerkin dissipation (INHALE_demo.ipynb cell 20) of u, v, w into out = (k_x, k_y,
    k_z); eps_k = 1e-3 as the notebook sets it (INH:867)."""
    Z, Y, X = _shape(u)
    keep = [_w(K) for K in (Kdif, Kx, Ky, Kz)]
    scratch = _Scratch.get_bytes(L.lib().hfm_ns_pg_scratch_bytes(Z, Y, X), u.device)
    L.call("hfm_ns_pg_dissipation", _p(u), _p(v), _p(w), _p(sigma), *(_p(t) for t in out), Z, Y, X,
           *(kk[1] for kk in keep), float(dt), float(eps_k), _p(scratch), _stream())
    return out


def pressure_gradient(p, u, v, w, Kx, Ky, Kz):
    """In place u -= pu(p), v -= pv(p), w -= pw(p)."""
    Z, Y, X = _shape(p)
    keep = [_w(K) for K in (Kx, Ky, Kz)]
    L.call("hfm_ns_pressure_gradient", _p(p), _p(u), _p(v), _p(w), Z, Y, X,
           *(k[1] for k in keep), _stream())
    return u, v, w


def divergence(u, v, w, b, Su, Sv, Sw, bc_source=True):
    Z, Y, X = _shape(u)
    keep = [_w(K) for K in (Su, Sv, Sw)]
    L.call("hfm_ns_divergence", _p(u), _p(v), _p(w), _p(b), Z, Y, X, *(k[1] for k in keep),
           int(bc_source), _stream())
    return b


def obstacle_mask(shape, n_boxes=24, footprint=(4, 16), height=(8, 40), sigma=1e5, seed=0,
                  device="cuda"):
    """Sigma mask of seeded axis-aligned boxes standing on the floor z = 0 (the reference
    reads the building mask from a missing mesh file, naiver_stokes_3D.py:560-564)."""
    Z, Y, X = shape
    rng = np.random.default_rng(seed)
    m = np.zeros(shape, np.float32)
    for _ in range(n_boxes):
        fx, fy = (int(v) for v in rng.integers(footprint[0], footprint[1] + 1, 2))
        h = int(rng.integers(height[0], height[1] + 1))
        x0 = int(rng.integers(X // 8, max(X // 8 + 1, X - fx - X // 8)))
        y0 = int(rng.integers(1, max(2, Y - fy - 1)))
        m[1:min(Z - 1, 1 + h), y0:y0 + fy, x0:x0 + fx] = sigma
    return torch.from_numpy(m).to(device)


def mask_from_mesh(mesh, shape, sigma=1e5, offset=16, device="cuda"):
    """Sigma mask from the reference's geometry array (``naiver_stokes_3D.py:527,560-564``):
    ``mesh`` has shape (1, X + 2 offset, Y + 2 offset, Z', 1) indexed [0][x + offset]
    [y + offset][z][0]; an interior cell (1 <= x, y, z <= extent - 2) whose mesh value is 0 is
    solid and gets ``sigma``, every other cell 0.  Returns a (Z, Y, X) float32 tensor."""
    Z, Y, X = shape
    m = np.asarray(mesh)[0, offset:offset + X, offset:offset + Y, :Z, 0]  # (X, Y, Z)
    solid = np.transpose(m == 0, (2, 1, 0))                               # (Z, Y, X)
    out = np.zeros(shape, np.float32)
    inner = (slice(1, Z - 1), slice(1, Y - 1), slice(1, X - 1))
    out[inner] = np.where(solid[inner], np.float32(sigma), np.float32(0))
    return torch.from_numpy(out).to(device)


def load_mesh_mask(path, shape, sigma=1e5, offset=16, device="cuda"):
    """``np.load`` of a reference mesh file (e.g. ``mesh_64_sk.npy``) and ``mask_from_mesh``."""
    return mask_from_mesh(np.load(path), shape, sigma, offset, device)


@dataclass
class NSConfig:
    dt: float = 0.1
    dx: float = 1.0
    Re: float = 0.25            # the reference's "Re" is the diffusion coefficient nu
    ub: float = 1.0
    diffusion: str = "27"       # "27" (reference w1) or "7" (7-point Laplacian)
    adv_factor: float = 1.0     # 0.5 in AI_HFM_v3.ipynb
    pressure: str = "reference" # "reference" (sawtooth, multi_itr cycles) or "fcycle"
    multi_itr: int = 10
    p_tol: float = 1e-5
    n_levels: int = 0           # 0: down to 2^3 (reference form)
    pg: bool = False            # Petrov-Galerkin dissipation instead of the diffusion stencil
    eps_k: float = 1e-3         #   (INHALE_demo.ipynb cells 20, 24; eps as INH:867)


def laplacian7(scale):
    K = np.zeros((3, 3, 3))
    K[1, 1, 1] = -6
    K[0, 1, 1] = K[2, 1, 1] = K[1, 0, 1] = K[1, 2, 1] = K[1, 1, 0] = K[1, 1, 2] = 1
    return (K * scale).astype(np.float32)


class NSStepper:
    """Fields u, v, w, p (Z, Y, X) and the immersed-body sigma on the device."""

    def __init__(self, shape, cfg=None, sigma=None, device="cuda"):
        self.cfg = cfg or NSConfig()
        c = self.cfg
        self.shape = tuple(shape)
        Z, Y, X = self.shape
        z = lambda: torch.zeros(self.shape, device=device)
        self.u, self.v, self.w, self.p = z(), z(), z(), z()
        self.bu, self.bv, self.bw = z(), z(), z()
        self.nu, self.nv, self.nw = z(), z(), z()
        self.rhs = z()
        self.kx, self.ky, self.kz = (z(), z(), z()) if self.cfg.pg else (None, None, None)
        self.sigma = sigma if sigma is not None else z()
        self.Kdif = (W.diffusion27(c.dt, c.Re, c.dx) if c.diffusion == "27"
                     else laplacian7(c.dt * c.Re / c.dx ** 2))
        self.Kx, self.Ky, self.Kz = W.advection(c.dt, c.dx, c.adv_factor)
        self.Su, self.Sv, self.Sw = W.divergence(c.dt, c.dx, c.adv_factor)
        self.Kp = W.pressure27(c.dx)
        levels = c.n_levels or int(np.log2(min(self.shape))) if c.pressure == "reference" else c.n_levels
        if c.pressure == "reference":
            pc = SolverConfig.reference(n_levels=levels, fine_smooth=False, zero_xend=True,
                                        cycles=10 ** 9)
            pc.cycles_per_launch = 2 * ((c.multi_itr + 1) // 2)
        else:
            pc = SolverConfig(cycle="F", accel="none", tol=c.p_tol, max_cycles=500,
                              n_levels=levels, min_coarse_edge=4, coarse_scale=0.5,
                              zero_xend=True, cycles_per_launch=2)
        self.pcfg = pc
        self.mg = Multigrid(self.shape, L.OP_K27, pc, slots=1)
        self.mg.set_operator(Stencil27(self.Kp))
        self.itime = 0
        self.p_cycles = []
        self.p_status = []  # per step: the pressure solve's status (0 = reached p_tol)
        self.p_rel = []     # and its relative residual
        # the reference's clock (naiver_stokes_3D.py:519-523, 549, 572): ctime_old is
        # nrestart * dt after a restart, and each step adds dt + ctime_old to ctime
        self.nrestart = 0
        self.ctime_old = 0.0
        self.ctime = 0.0

    def close(self):
        self.mg.close()

    def _pressure_solve(self):
        c = self.cfg
        if c.pressure == "reference":
            self.mg.load(0, self.rhs, self.p)
            self.mg.run(c.multi_itr)
            self.mg.fetch(0, self.p)
            self.p_cycles.append(c.multi_itr)
            self.p_status.append(L.OK)  # a fixed cycle count, no tolerance (as the reference)
            self.p_rel.append(float("nan"))
        else:
            self.mg.load(0, self.rhs, self.p)
            while True:
                self.mg.run(self.pcfg.cycles_per_launch)
                st = self.mg.query()[0]
                if not st["active"]:
                    break
            self.mg.fetch(0, self.p)
            self.p_cycles.append(st["cycles"])
            self.p_status.append(st["status"])
            self.p_rel.append(st["rel_resid"])

    def step(self):
        """One time step in the reference's order (naiver_stokes_3D.py:571-727)."""
        c = self.cfg
        u, v, w, p = self.u, self.v, self.w, self.p
        boundary_condition_velocity(u, v, w, c.ub)
        boundary_condition_pressure(p)
        b, n = (self.bu, self.bv, self.bw), (self.nu, self.nv, self.nw)
        if c.pg:  # INHALE_demo.ipynb cell 24
            k = (self.kx, self.ky, self.kz)
            pg_dissipation(u, v, w, self.sigma, k, self.Kdif, self.Kx, self.Ky, self.Kz, c.dt, c.eps_k)
            momentum_stage_pg((u, v, w), (u, v, w), b, k, self.Kx, self.Ky, self.Kz, 0.5)
            boundary_condition_velocity(*b, c.ub)
            pg_dissipation(*b, self.sigma, k, self.Kdif, self.Kx, self.Ky, self.Kz, c.dt, c.eps_k)
            momentum_stage_pg(b, (u, v, w), n, k, self.Kx, self.Ky, self.Kz, 1.0)
        else:
            momentum_stage((u, v, w), (u, v, w), b, self.Kdif, self.Kx, self.Ky, self.Kz, 0.5)
            boundary_condition_velocity(*b, c.ub)
            momentum_stage(b, (u, v, w), n, self.Kdif, self.Kx, self.Ky, self.Kz, 1.0)
        self.u, self.nu = self.nu, self.u
        self.v, self.nv = self.nv, self.v
        self.w, self.nw = self.nw, self.w
        u, v, w = self.u, self.v, self.w
        bluff_body(u, v, w, self.sigma, c.dt)
        pressure_gradient(p, u, v, w, self.Kx, self.Ky, self.Kz)
        boundary_condition_velocity(u, v, w, c.ub)
        divergence(u, v, w, self.rhs, self.Su, self.Sv, self.Sw, bc_source=True)
        self._pressure_solve()
        boundary_condition_pressure(p)
        pressure_gradient(p, u, v, w, self.Kx, self.Ky, self.Kz)
        boundary_condition_velocity(u, v, w, c.ub)
        bluff_body(u, v, w, self.sigma, c.dt)
        self.ctime = self.ctime + c.dt + self.ctime_old
        self.itime += 1

    # reference checkpoint layout: u, v, w, p saved as (Z, Y, X) float32 .npy files named
    # <field><step> (save_data, naiver_stokes_3D.py:488-497; restart :531-549)
    def save(self, directory, itime=None, n_out=None):
        """Write u, v, w, p as ``u<itime>.npy`` ... in ``directory``.  ``itime`` defaults to
        the steps taken so far; with ``n_out`` the files are written only when ``itime`` is a
        multiple of it, as ``save_data`` does.  Returns True when files were written."""
        it = self.itime if itime is None else itime
        if n_out is not None and it % n_out != 0:
            return False
        os.makedirs(directory, exist_ok=True)
        for name in ("u", "v", "w", "p"):
            np.save(os.path.join(directory, "%s%d.npy" % (name, it)),
                    getattr(self, name).cpu().numpy())
        return True

    def restart(self, directory, itime):
        """Read ``u<itime>.npy`` ... (cast to float32) into the fields and continue from step
        ``itime``: nrestart = itime, ctime_old = nrestart * dt (naiver_stokes_3D.py:531-549)."""
        arrays = {}
        for name in ("u", "v", "w", "p"):
            a = np.load(os.path.join(directory, "%s%d.npy" % (name, itime))).astype(np.float32)
            if a.shape != self.shape:
                raise ValueError("%s%d.npy has shape %s, the stepper %s" % (name, itime, a.shape, self.shape))
            arrays[name] = a
        for name, a in arrays.items():
            getattr(self, name).copy_(torch.from_numpy(a))
        self.itime = itime
        self.nrestart = itime
        self.ctime_old = itime * self.cfg.dt

    def max_divergence(self):
        b = torch.empty_like(self.u)
        divergence(self.u, self.v, self.w, b, self.Su, self.Sv, self.Sw, bc_source=False)
        return float(b.abs().max())


def config1_run(steps=1000, shape=(64, 128, 128), seed=0, log_every=100):
    """Flow past 24 seeded box obstacles on a 128 x 128 x 64 grid (x the flow direction, z up):
    dx = 1, nu = 0.05, dt = 0.5, 7-point diffusion, smoothed central advection, sigma-penalty
    mask, pressure by F(2,2) cycles to 1e-5 per step.  Returns timings and
    diagnostics."""
    import time
    cfg = NSConfig(dt=0.5, dx=1.0, Re=0.05, ub=1.0, diffusion="7", pressure="fcycle", p_tol=1e-5)
    sig = obstacle_mask(shape, n_boxes=24, footprint=(4, 16), height=(8, 40), sigma=1e5, seed=seed)
    st = NSStepper(shape, cfg, sigma=sig)
    try:
        st.step()
        torch.cuda.synchronize()
        hist = []
        t0 = time.perf_counter()
        for k in range(1, steps):
            st.step()
            if k % log_every == 0:
                hist.append({"step": k, "max_u": float(st.u.abs().max()),
                             "p_cycles": st.p_cycles[-1]})
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        return {"shape": list(shape), "steps": steps, "seconds": dt, "ms_per_step": 1e3 * dt / max(steps - 1, 1),
                "mean_p_cycles": float(np.mean(st.p_cycles)), "max_abs_div": st.max_divergence(),
                "finite": bool(torch.isfinite(st.u).all()), "history": hist}
    finally:
        st.close()
