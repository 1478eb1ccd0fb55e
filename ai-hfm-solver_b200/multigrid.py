"""Multigrid solver handle over ``libhfm`` (``hfm_mg_*``).

``SolverConfig`` holds the knobs the reference keeps as module-level constants
(``multi_itr``, ``j_itr``, the level list and the Jacobi diagonal,
``Anisotropic_3d_Multigrid_7point.ipynb:402-405``) plus the textbook cycle parameters of the
solver configurations.  ``Multigrid`` owns the resident hierarchy of ``slots`` same-size
instances; slots are loaded, advanced together by CUDA graphs of whole cycles, polled and
fetched independently, which is what the serving layer builds on.
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib as L
from .ops import Operator, _check_field, _stream

_CYCLES = {"sawtooth": L.CYCLE_SAWTOOTH, "V": L.CYCLE_V, "F": L.CYCLE_F}
_ACCEL = {None: L.ACCEL_NONE, "none": L.ACCEL_NONE, "cg": L.ACCEL_CG, "ir": L.ACCEL_IR}
_STORAGE = {"f32": L.F32, "bf16": L.BF16, "f16": L.F16}


@dataclass
class SolverConfig:
    cycle: str = "V"            # "sawtooth" (reference), "V" or "F"
    accel: str = "none"         # "none" (stationary cycles), "cg" (cycle preconditions CG) or
                                # "ir" (float64 iterative refinement around CG)
    n_levels: int = 0           # 0: halve while every extent is even and > min_coarse_edge
    min_coarse_edge: int = 4
    nu_pre: int = 2
    nu_post: int = 2
    coarse_sweeps: int = 32
    omega: float = 2.0 / 3.0
    coarse_omega: float = 2.0 / 3.0
    coarse_scale: float = 0.5   # operator on level l scaled by coarse_scale**l (1 = reference)
    sawtooth_fine_smooth: bool = True
    top_copy: bool = False      # boundary_condition_top after each reference cycle
    zero_xend: bool = False     # NS pressure form: r and phi zero on x = X-1
    storage: str = "f32"
    tol: float = 1e-6
    max_cycles: int = 500
    cycles_per_launch: int = 4
    inner_tol: float = 1e-6     # "ir": inner CG stops at max(inner_tol ||r0||, 0.3 tol ||b||)
    inner_max_cycles: int = 200
    fused_coarse: bool = True   # deep V-cycle levels (<= 4096 cells) in one fused kernel
    fused_pre: bool = True      # first two pre-sweeps from zero in one pass (SIGMA7, TMA levels)
    faces: bool = True          # 16-bit SIGMA7: face-coefficient kernels on the TMA levels
    persistent: bool = False    # small end of the V-cycle as one persistent kernel (>= 8 slots)
    temporal: bool = False      # two Jacobi sweeps per pass on FACE7 levels (16-bit storage)
    sawtooth_coarse_sweeps: int = 1  # Jacobi sweeps on the sawtooth's coarsest level (1 =
                                     # Anisotropic_3d_Multigrid_7point.ipynb; 2 = the serial
                                     # run of parallel_multigrid_advection_diffusion_3D.ipynb)

    @staticmethod
    def reference(n_levels, fine_smooth=True, top_copy=False, zero_xend=False, cycles=1000,
                  coarse_sweeps=1):
        """The reference sawtooth cycle: omega 1, one Jacobi per level, same operator on every
        level (``Anisotropic_3d_Multigrid_7point.ipynb:402-449``); ``coarse_sweeps`` Jacobi
        sweeps on the coarsest level."""
        return SolverConfig(cycle="sawtooth", n_levels=n_levels, nu_pre=0, nu_post=1,
                            omega=1.0, coarse_omega=1.0, coarse_scale=1.0,
                            sawtooth_fine_smooth=fine_smooth, top_copy=top_copy,
                            zero_xend=zero_xend, tol=1e-300, max_cycles=cycles,
                            cycles_per_launch=2, sawtooth_coarse_sweeps=coarse_sweeps)

    def struct(self, op_kind):
        c = L.HfmMgConfig()
        L.lib().hfm_mg_config_default(C.byref(c))
        c.op_kind = op_kind
        c.cycle = _CYCLES[self.cycle]
        c.accel = _ACCEL[self.accel]
        c.n_levels = self.n_levels
        c.min_coarse_edge = self.min_coarse_edge
        c.nu_pre, c.nu_post = self.nu_pre, self.nu_post
        c.coarse_sweeps = self.coarse_sweeps
        c.omega, c.coarse_omega = self.omega, self.coarse_omega
        c.coarse_scale = self.coarse_scale
        c.sawtooth_fine_smooth = int(self.sawtooth_fine_smooth)
        c.flags = (L.FLAG_TOP_COPY if self.top_copy else 0) | (L.FLAG_ZERO_XEND if self.zero_xend else 0)
        c.storage = _STORAGE[self.storage]
        c.tol = self.tol
        c.max_cycles = self.max_cycles
        c.cycles_per_launch = self.cycles_per_launch
        c.inner_tol = self.inner_tol
        c.inner_max_cycles = self.inner_max_cycles
        c.options = (0 if self.fused_coarse else L.OPT_NO_FUSED_COARSE) | \
            (0 if self.fused_pre else L.OPT_NO_FUSED_PRE) | \
            (0 if self.faces else L.OPT_NO_FACES) | \
            (L.OPT_PERSISTENT if self.persistent else 0) | \
            (L.OPT_TEMPORAL if self.temporal else 0)
        if self.cycle == "sawtooth" and self.sawtooth_coarse_sweeps != 1:
            c.options |= L.OPT_SAWTOOTH_COARSE_SWEEPS
            c.coarse_sweeps = self.sawtooth_coarse_sweeps
        return c


def footprint_bytes(cfg, op_kind, shape, slots):
    s = cfg.struct(op_kind)
    return int(L.lib().hfm_mg_footprint_bytes(C.byref(s), shape[0], shape[1], shape[2], slots))


class Multigrid:
    """Resident multigrid hierarchy for ``slots`` instances of extent ``shape`` (Z, Y, X)."""

    def __init__(self, shape, op_kind, cfg=None, slots=1):
        self.cfg = cfg or SolverConfig()
        self.shape = tuple(int(v) for v in shape)
        self.slots = int(slots)
        self.op_kind = op_kind
        self._s = self.cfg.struct(op_kind)
        h = C.c_void_p()
        Z, Y, X = self.shape
        L.call("hfm_mg_create", C.byref(self._s), Z, Y, X, self.slots, C.byref(h))
        self._h = h
        self._stats = (L.HfmSlotStats * self.slots)()

    # ------------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            torch.cuda.synchronize()
            L.lib().hfm_mg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------ queries
    @property
    def levels(self):
        out = []
        for l in range(L.lib().hfm_mg_num_levels(self._h)):
            z, y, x = C.c_int(), C.c_int(), C.c_int()
            L.call("hfm_mg_level_shape", self._h, l, C.byref(z), C.byref(y), C.byref(x))
            out.append((z.value, y.value, x.value))
        return out

    # ------------------------------------------------------------------ slots
    def set_operator(self, op, slot=-1):
        """Install the fine operator (and its coefficient hierarchy) for ``slot`` (-1: all;
        SIGMA7 coefficient tensors then hold every slot, ``(slots, Z, Y, X)``)."""
        if not isinstance(op, Operator):
            raise TypeError("op must be an ops.Operator")
        s = op.struct()
        self._op_keep = op
        L.call("hfm_mg_set_operator", self._h, int(slot), C.byref(s), _stream())

    def load(self, slot, rhs, phi0=None):
        _check_field(rhs, "rhs")
        if phi0 is not None:
            _check_field(phi0, "phi0")
        L.call("hfm_mg_load", self._h, int(slot), C.c_void_p(rhs.data_ptr()),
               C.c_void_p(phi0.data_ptr() if phi0 is not None else 0), _stream())

    def run(self, cycles):
        L.call("hfm_mg_run", self._h, int(cycles), _stream())

    def query(self):
        L.call("hfm_mg_query", self._h, self._stats, _stream())
        return [dict(active=s.active, status=s.status, cycles=s.cycles, outer=s.outer,
                     norm_b=s.norm_b, rel_resid=s.rel_resid) for s in self._stats]

    def query_async(self, host_buf):
        """Enqueue a copy of all slots' statistics into ``host_buf`` (pinned uint8 tensor of
        ``slots * sizeof(HfmSlotStats)`` bytes); decode with ``decode_stats`` once the stream
        has passed this point."""
        L.call("hfm_mg_query_async", self._h, C.c_void_p(host_buf.data_ptr()), _stream())

    def decode_stats(self, host_buf):
        arr = (L.HfmSlotStats * self.slots).from_address(host_buf.data_ptr())
        return [dict(active=s.active, status=s.status, cycles=s.cycles, outer=s.outer,
                     norm_b=s.norm_b, rel_resid=s.rel_resid) for s in arr]

    def fetch(self, slot, out=None):
        out = torch.empty(self.shape, dtype=torch.float32, device="cuda") if out is None else out
        L.call("hfm_mg_fetch", self._h, int(slot), C.c_void_p(out.data_ptr()), _stream())
        return out

    def load_f64(self, slot, rhs, phi0=None):
        """float64 right-hand side / initial guess (accel="ir")."""
        for t in (rhs, phi0):
            if t is not None and (t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous()):
                raise TypeError("load_f64 takes contiguous float64 CUDA tensors")
        L.call("hfm_mg_load_f64", self._h, int(slot), C.c_void_p(rhs.data_ptr()),
               C.c_void_p(phi0.data_ptr() if phi0 is not None else 0), _stream())

    def fetch_f64(self, slot, out=None):
        out = torch.empty(self.shape, dtype=torch.float64, device="cuda") if out is None else out
        L.call("hfm_mg_fetch_f64", self._h, int(slot), C.c_void_p(out.data_ptr()), _stream())
        return out

    def cancel(self, slot):
        L.call("hfm_mg_cancel", self._h, int(slot), _stream())

    def read_level(self, slot, level, which):
        shp = self.levels[level]
        out = torch.empty(shp, dtype=torch.float32, device="cuda")
        L.call("hfm_mg_read_level", self._h, int(slot), int(level), int(which),
               C.c_void_p(out.data_ptr()), _stream())
        return out

    def solve(self, rhs):
        """Solve every slot for ``rhs`` of shape ``(slots, Z, Y, X)``; returns (phi, stats).
        A slot that does not reach tolerance, meets NaN or sees an expired device wait keeps
        its status in stats (no exception)."""
        _check_field(rhs, "rhs")
        phi = torch.empty_like(rhs)
        st = L.lib().hfm_mg_solve(self._h, C.c_void_p(rhs.data_ptr()), C.c_void_p(phi.data_ptr()),
                                  self._stats, _stream())
        if st not in (L.OK, L.ERR_NOT_CONVERGED, L.ERR_NAN, L.ERR_TIMEOUT):
            L.check(st, "hfm_mg_solve")
        stats = [dict(active=s.active, status=s.status, cycles=s.cycles, outer=s.outer,
                      norm_b=s.norm_b, rel_resid=s.rel_resid) for s in self._stats]
        return phi, stats


def precision_check(n=256, log_std=2.0, seed=0, tol=1e-10, storages=("bf16", "f16", "f32"),
                    oracle_error=False):
    """The precision workload: the anisotropic operator at ``n``^3 with sigma log-std
    ``log_std`` solved by float64 iterative refinement around CG preconditioned by V(2,2)
    cycles stored in each of ``storages``.  Reports per storage the cycles, refinement steps,
    float64 relative residual, time and - with ``oracle_error`` - the error against a float64
    solve of the same system (float64 refinement driven to 1e-13 with float32 inner cycles)."""
    import time
    from . import problems, ops
    sig = problems.anisotropic_sigma((n, n, n), seed=seed, log_std=log_std)
    f = problems.dipole((n, n, n), seed=seed)
    sd = torch.from_numpy(sig).cuda()
    fd = torch.from_numpy(f.astype(np.float64)).cuda()
    op = ops.Sigma7(sd[0], sd[1], sd[2])

    def run(storage, t):
        cfg = SolverConfig(cycle="V", accel="ir", storage=storage, tol=t, max_cycles=2000)
        with Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=1) as h:
            h.set_operator(op)
            h.load_f64(0, fd)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            while True:
                h.run(8)
                st = h.query()[0]
                if not st["active"]:
                    break
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            return h.fetch_f64(0), st, dt

    ref = run("f32", 1e-13)[0] if oracle_error else None
    out = {}
    for s in storages:
        x, st, dt = run(s, tol)
        d = {"status": st["status"], "cycles": st["cycles"], "outer": st["outer"],
             "rel_resid": st["rel_resid"], "seconds": dt}
        if ref is not None:
            d["error_vs_f64"] = float((x - ref).norm() / ref.norm())
        out[s] = d
    return out
