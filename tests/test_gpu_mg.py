"""GPU parity of the multigrid handle (hfm_mg_* through the C ABI) against the oracle.

Reference-mode (sawtooth) parity: float32 fields within 1e-5 relative (to the field max) of
the float32 oracle after 1, 2, 3 and 10 cycles.  Config-mode cycles: same bar per cycle;
solves: relative residual below tol, error against the float64 oracle stated.
"""
import os

import numpy as np
import pytest

from oracle import mg, weights as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def close(got, ref, rtol=1e-5):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    err = np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-30)
    assert err <= rtol, "max rel err %.3e > %.1e" % (err, rtol)
    return err


@pytest.fixture(scope="module")
def T(hfm):
    import torch
    return torch


def dev(T, a):
    return T.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def run_sawtooth(hfm, T, K, b, phi0, n_levels, cycles, **kw):
    M = hfm.multigrid
    cfg = M.SolverConfig.reference(n_levels=n_levels, cycles=cycles + 2, **kw)
    with M.Multigrid(b.shape, hfm._lib.OP_K27, cfg, slots=1) as h:
        h.set_operator(hfm.ops.Stencil27(K))
        h.load(0, dev(T, b), dev(T, phi0))
        outs = []
        for _ in range(cycles // 2):
            h.run(2)
            outs.append(h.fetch(0).cpu().numpy())
        return outs, h.levels


def test_sawtooth_7point_golden(hfm, T):
    g = np.load(os.path.join(GOLD, "oracle_small.npz"))
    b = g["saw7_b"]
    M = hfm.multigrid
    cfg = M.SolverConfig.reference(n_levels=5, cycles=10)
    cfg.cycles_per_launch = 1
    with M.Multigrid(b.shape, hfm._lib.OP_K27, cfg, slots=1) as h:
        h.set_operator(hfm.ops.Stencil27(W.w2_7point()))
        assert h.levels == [(16, 16, 16), (8, 8, 8), (4, 4, 4), (2, 2, 2), (1, 1, 1)]
        h.load(0, dev(T, b), dev(T, b))
        h.run(2)
        close(h.fetch(0).cpu(), g["saw7_after_2"])


def test_sawtooth_7point_10_cycles_and_levels(hfm, T):
    """7point.ipynb cycle on 32^3 (6 levels down to 1^3): fields and per-level w after
    10 cycles."""
    n = 32
    b = np.zeros((n, n, n), np.float32)
    b[11:21, 11:21, 11:21] = 1.0
    K = W.w2_7point()
    ops = mg.hierarchy(mg.Stencil27(K), 6)
    ref = b.copy()
    refs = []
    keep = {}
    for c in range(10):
        ref = mg.sawtooth_cycle(ops, ref, b, keep=keep)
        refs.append(ref)
    M = hfm.multigrid
    cfg = M.SolverConfig.reference(n_levels=6, cycles=20)
    with M.Multigrid(b.shape, hfm._lib.OP_K27, cfg, slots=1) as h:
        h.set_operator(hfm.ops.Stencil27(K))
        h.load(0, dev(T, b), dev(T, b))
        for k in range(5):
            h.run(2)
            close(h.fetch(0).cpu(), refs[2 * k + 1])
        # the last cycle's corrections and residuals, level by level
        for l in range(1, 6):
            close(h.read_level(0, l, 0).cpu(), keep["w"][l], rtol=1e-4)
            close(h.read_level(0, l, 1).cpu(), keep["r"][l], rtol=1e-4)


@pytest.mark.parametrize("n", [16, 64])
def test_sawtooth_neumann_top(hfm, T, n):
    """Anisotropic_3d_Multigrid_7point_BC.ipynb: boundary_condition_top after each cycle."""
    b = np.zeros((n, n, n), np.float32)
    b[n // 3:n // 2, n // 3:n // 2, n // 3:n // 2] = 1.0
    K = W.w2_7point()
    nl = int(np.log2(n)) + 1
    ops = mg.hierarchy(mg.Stencil27(K), nl)
    ref = b.copy()
    for _ in range(4):
        ref = mg.sawtooth_cycle(ops, ref, b, top_copy=True)
    outs, _ = run_sawtooth(hfm, T, K, b, b, nl, 4, top_copy=True)
    close(outs[-1], ref)
    np.testing.assert_array_equal(outs[-1][0], outs[-1][1])


def test_sawtooth_ns_pressure_golden(hfm, T):
    """naiver_stokes_3D.py:646-703 pressure cycle: 27-point w5, coarsest 2^3, no fine-level
    Jacobi on w, residual and pressure zeroed on x = X-1."""
    g = np.load(os.path.join(GOLD, "oracle_small.npz"))
    pb = g["sawns_b"]
    outs, levels = run_sawtooth(hfm, T, W.w5_pressure27(), pb, np.zeros_like(pb), 4, 2,
                                fine_smooth=False, zero_xend=True)
    assert levels[-1] == (2, 2, 2)
    close(outs[-1], g["sawns_after_2"])


def test_sawtooth_rectangular(hfm, T):
    """Anisotropic_3d_Multigrid_7point_BC_Rec.ipynb: (nz, ny, nx) = (5*m, m, m) grids with
    dz = 5 coarsen to a 5x1x1 coarsest level."""
    b = np.zeros((40, 8, 8), np.float32)
    b[10:20, 2:6, 2:6] = 1.0
    K = W.w2_7point(dz=5.0)
    ops = mg.hierarchy(mg.Stencil27(K), 4)
    ref = b.copy()
    for _ in range(2):
        ref = mg.sawtooth_cycle(ops, ref, b)
    outs, levels = run_sawtooth(hfm, T, K, b, b, 4, 2)
    assert levels[-1] == (5, 1, 1)
    close(outs[-1], ref)


def _problem(hfm, n, seed, log_std=1.0):
    sig = hfm.problems.anisotropic_sigma((n, n, n), seed=seed, log_std=log_std)
    f = hfm.problems.dipole((n, n, n), seed=seed)
    return sig, f


@pytest.mark.parametrize("cycle,n", [("V", 32), ("F", 32), ("V", 64)])
def test_config_cycles_match_oracle(hfm, T, cycle, n):
    sig, f = _problem(hfm, n, 5)
    oop = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float32)
    shapes = mg.level_shapes((n, n, n))
    ops = mg.hierarchy(oop, len(shapes), 0.5)
    ccfg = mg.CycleConfig(2, 2, 2.0 / 3.0, 32)
    M = hfm.multigrid
    cfg = M.SolverConfig(cycle=cycle, tol=1e-300, max_cycles=50, cycles_per_launch=1)
    with M.Multigrid((n, n, n), hfm._lib.OP_SIGMA7, cfg, slots=1) as h:
        assert h.levels == shapes
        h.set_operator(hfm.ops.Sigma7(*(dev(T, sig[k]) for k in range(3))))
        h.load(0, dev(T, f))
        ref = np.zeros_like(f)
        fn = mg.vcycle if cycle == "V" else mg.fcycle
        for c in range(3):
            ref = fn(ops, 0, ref, f, ccfg)
            h.run(1)
            close(h.fetch(0).cpu(), ref)


@pytest.mark.parametrize("accel,cycle,n", [("cg", "V", 32), ("none", "V", 32), ("none", "F", 32),
                                           ("cg", "V", 64)])
def test_solve_to_tolerance(hfm, T, accel, cycle, n):
    sig, f = _problem(hfm, n, 6)
    M = hfm.multigrid
    cfg = M.SolverConfig(cycle=cycle, accel=accel, tol=1e-6, max_cycles=1000)
    with M.Multigrid((n, n, n), hfm._lib.OP_SIGMA7, cfg, slots=1) as h:
        h.set_operator(hfm.ops.Sigma7(*(dev(T, sig[k]) for k in range(3))))
        phi, st = h.solve(dev(T, f[None]))
    assert st[0]["status"] == 0, st
    oop = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float64)
    p = phi[0].double().cpu().numpy()
    rel = mg.rel_residual(oop, p, f)
    assert rel < 1.5e-6
    assert abs(rel - st[0]["rel_resid"]) < 1e-6
    if n <= 32:
        # error against the float64 oracle solution of the same discrete system
        ops64 = mg.hierarchy(oop, len(mg.level_shapes((n, n, n))), 0.5)
        x64, _ = mg.pcg_solve(ops64, f.astype(np.float64), mg.CycleConfig(), tol=1e-11)
        err = np.linalg.norm(p - x64) / np.linalg.norm(x64)
        assert err < 1e-3, err


def test_slots_alone_and_in_the_mix(hfm, T):
    """Each slot's result is identical whether it is solved alone or with others."""
    n = 16
    M = hfm.multigrid
    cfg = M.SolverConfig(cycle="V", accel="cg", tol=1e-6)
    probs = [_problem(hfm, n, s, 0.5 + 0.5 * s) for s in range(3)]
    sig = np.stack([p[0] for p in probs], axis=1)  # (3, slots, n, n, n)
    f = np.stack([p[1] for p in probs])
    with M.Multigrid((n, n, n), hfm._lib.OP_SIGMA7, cfg, slots=3) as h:
        h.set_operator(hfm.ops.Sigma7(*(dev(T, sig[k]) for k in range(3))))
        phi, st = h.solve(dev(T, f))
        mix = phi.cpu().numpy()
    for s in range(3):
        with M.Multigrid((n, n, n), hfm._lib.OP_SIGMA7, cfg, slots=1) as h:
            h.set_operator(hfm.ops.Sigma7(*(dev(T, sig[k, s]) for k in range(3))))
            phi1, st1 = h.solve(dev(T, f[s:s + 1]))
        assert st1[0]["cycles"] == st[s]["cycles"]
        np.testing.assert_array_equal(phi1[0].cpu().numpy(), mix[s])


def test_failure_statuses(hfm, T):
    n = 16
    sig, f = _problem(hfm, n, 8)
    M, L = hfm.multigrid, hfm._lib
    cfg = M.SolverConfig(cycle="V", tol=1e-12, max_cycles=2)
    with M.Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=3) as h:
        h.set_operator(hfm.ops.Sigma7(*(dev(T, np.broadcast_to(sig[k], (3, n, n, n))) for k in range(3))))
        bad = f.copy()
        bad[3, 3, 3] = np.nan
        rhs = np.stack([f, bad, np.zeros_like(f)])
        phi, st = h.solve(dev(T, rhs))
    assert st[0]["status"] == L.ERR_NOT_CONVERGED and st[0]["cycles"] == 2
    assert st[1]["status"] == L.ERR_NAN
    assert st[2]["status"] == L.OK and np.all(phi[2].cpu().numpy() == 0)


def test_cancel_frees_slot(hfm, T):
    n = 16
    sig, f = _problem(hfm, n, 9)
    M = hfm.multigrid
    cfg = M.SolverConfig(cycle="V", accel="cg", tol=1e-6)
    with M.Multigrid((n, n, n), hfm._lib.OP_SIGMA7, cfg, slots=1) as h:
        h.set_operator(hfm.ops.Sigma7(*(dev(T, sig[k]) for k in range(3))))
        h.load(0, dev(T, f))
        h.run(1)
        h.cancel(0)
        assert h.query()[0]["active"] == 0
        phi, st = h.solve(dev(T, f[None]))
        assert st[0]["status"] == 0


def test_ns_pressure_form_64(hfm, T):
    """NS pressure cycle on 64^3 (27-point operator, x-end zeroing) through the large-grid
    kernels."""
    rng = np.random.default_rng(21)
    n = 64
    pb = rng.standard_normal((n, n, n)).astype(np.float32)
    K = W.w5_pressure27()
    ops27 = mg.hierarchy(mg.Stencil27(K), 6)
    p = np.zeros_like(pb)
    for _ in range(2):
        p = mg.sawtooth_cycle(ops27, p, pb, fine_smooth=False, zero_xend=True)
    outs, _ = run_sawtooth(hfm, T, K, pb, np.zeros_like(pb), 6, 2, fine_smooth=False, zero_xend=True)
    close(outs[-1], p)


def test_no_device_timeouts(hfm, T):
    import ctypes as C
    cnt = C.c_int(-1)
    hfm._lib.call("hfm_device_timeouts", C.byref(cnt), 0)
    assert cnt.value == 0


@pytest.mark.parametrize("n", [16, 64])
def test_fcycle_with_outflow_rule_matches_oracle(hfm, T, n):
    """F(2,2) cycles on the 27-point pressure operator with the NS outflow rule (x = X-1
    pinned to zero on the fine level), as the pressure solve of the NS stepper."""
    rng = np.random.default_rng(41)
    b = rng.standard_normal((n, n, n)).astype(np.float32)
    K = W.w5_pressure27()
    shapes = mg.level_shapes((n, n, n))
    ops = mg.hierarchy(mg.Stencil27(K), len(shapes), 0.5)
    ccfg = mg.CycleConfig(2, 2, 2.0 / 3.0, 32, zero_xend=True)
    M = hfm.multigrid
    cfg = M.SolverConfig(cycle="F", tol=1e-300, max_cycles=50, cycles_per_launch=1, zero_xend=True)
    with M.Multigrid((n, n, n), hfm._lib.OP_K27, cfg, slots=1) as h:
        h.set_operator(hfm.ops.Stencil27(K))
        h.load(0, dev(T, b))
        ref = np.zeros_like(b)
        for _ in range(3):
            ref = mg.fcycle(ops, 0, ref, b, ccfg)
            h.run(1)
            got = h.fetch(0).cpu().numpy()
            close(got[..., :-1], ref[..., :-1])


def test_sawtooth_directional_nonuniform_mesh(hfm, T):
    """BGS_multigrid_v1.ipynb: the six-array directional operator on the stretched mesh of
    cells 34-38 (sizes grow from the centre in x and y and along z), coefficient hierarchy by
    restriction (cell 38), reference sawtooth cycle (cell 42), against the oracle."""
    ops = hfm.ops
    shape = (40, 32, 32)
    mx, my, mz = ops.bgs_mesh(shape)
    gop = ops.dir7_from_mesh(100.0, mx, my, mz)
    arrs = {k: v.cpu().numpy() for k, v in zip(gop.ORDER, gop.A)}
    oop = mg.Dir7({k: v for k, v in arrs.items() if k != "tot"}, arrs["tot"], np.float32)
    # the product's coefficients are the oracle's cell-38 formula
    ref = mg.bgs_coefficients(100.0, mx, my, mz, ops.bgs_mesh_p1(mx, 2), ops.bgs_mesh_p1(my, 1),
                              ops.bgs_mesh_p1(mz, 0))
    for k in mg.Dir7.ORDER:
        np.testing.assert_allclose(arrs[k], ref[k], rtol=1e-6)
    b = np.zeros(shape, np.float32)
    b[10:20, 12:20, 12:20] = 1.0
    n_levels = 4  # 40x32x32 .. 5x4x4, exact halvings as in the reference's 640x128x128 case
    hier = mg.hierarchy(oop, n_levels)
    refv = b.copy()
    for _ in range(4):
        refv = mg.sawtooth_cycle(hier, refv, b)
    M = hfm.multigrid
    cfg = M.SolverConfig.reference(n_levels=n_levels, cycles=10)
    with M.Multigrid(shape, hfm._lib.OP_DIR7, cfg, slots=1) as h:
        h.set_operator(gop)
        h.load(0, dev(T, b), dev(T, b))
        h.run(2)
        h.run(2)
        close(h.fetch(0).cpu(), refv)


def test_directional_cg_solve(hfm, T):
    """The directional form in a config-mode solve: PCG with V(2,2) on the stretched mesh
    reaches 1e-6 measured by the float64 oracle."""
    ops = hfm.ops
    shape = (32, 32, 32)
    gop = ops.dir7_from_mesh(100.0, *ops.bgs_mesh(shape))
    f = hfm.problems.dipole(shape, seed=9)
    M = hfm.multigrid
    cfg = M.SolverConfig(cycle="V", accel="cg", tol=1e-6, max_cycles=500)
    with M.Multigrid(shape, hfm._lib.OP_DIR7, cfg, slots=1) as h:
        h.set_operator(gop)
        phi, st = h.solve(dev(T, f[None]))
    assert st[0]["status"] == 0, st
    arrs = {k: v.double().cpu().numpy() for k, v in zip(gop.ORDER, gop.A)}
    oop = mg.Dir7({k: v for k, v in arrs.items() if k != "tot"}, arrs["tot"], np.float64)
    assert mg.rel_residual(oop, phi[0].double().cpu().numpy(), f) < 1.5e-6


@pytest.mark.parametrize("cycle,storage", [("V", "f32"), ("F", "f32"), ("V", "bf16")])
def test_fused_coarse_cycle_matches_separate_kernels(hfm, T, cycle, storage):
    """The deep levels (<= 4096 cells) run as one fused kernel by default; the same cycles
    with every level launched separately (HFM_OPT_NO_FUSED_COARSE) give the same iterate to
    float32 rounding (float32 storage) or to the storage rounding the separate kernels add
    between sweeps (bf16)."""
    sig, f = _problem(hfm, 32, 8)
    M = hfm.multigrid
    outs = []
    for fused in (True, False):
        cfg = M.SolverConfig(cycle=cycle, storage=storage, tol=1e-300, max_cycles=10,
                             cycles_per_launch=1, fused_coarse=fused)
        # 8 instances: the fused path runs from 8 instances per handle up
        with M.Multigrid((32, 32, 32), hfm._lib.OP_SIGMA7, cfg, slots=8) as h:
            for s in range(8):
                h.set_operator(hfm.ops.Sigma7(*(dev(T, sig[k]) for k in range(3))), slot=s)
                h.load(s, dev(T, f))
            h.run(3)
            outs.append([h.fetch(s).cpu().numpy() for s in (0, 7)])
    close(outs[0][0], outs[1][0], rtol=1e-5 if storage == "f32" else 2e-2)
    np.testing.assert_array_equal(outs[0][0], outs[0][1])
    if cycle == "V" and storage == "f32":
        # and the fused path against the oracle's V-cycles directly
        oop = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float32)
        ops_ = mg.hierarchy(oop, len(mg.level_shapes((32, 32, 32))), 0.5)
        ref = np.zeros_like(f)
        for _ in range(3):
            ref = mg.vcycle(ops_, 0, ref, f, mg.CycleConfig(2, 2, 2.0 / 3.0, 32))
        close(outs[0][0], ref)


@pytest.mark.parametrize("storage", ["f32", "bf16", "f16"])
def test_fused_presmoothing_matches_two_sweeps(hfm, T, storage):
    """The first two pre-sweeps from zero run as one pass on TMA levels (phi1 = omega f / diag
    formed where the second sweep reads phi); against two separate sweeps
    (HFM_OPT_NO_FUSED_PRE) the iterate agrees to float32 rounding (float32 storage) or to the
    rounding of phi1 that the two-pass path stores (16-bit)."""
    shape = (32, 48, 64)
    sig = hfm.problems.anisotropic_sigma(shape, seed=11, log_std=1.0)
    f = hfm.problems.dipole(shape, seed=11)
    M = hfm.multigrid
    outs = []
    for fused in (True, False):
        cfg = M.SolverConfig(cycle="V", storage=storage, tol=1e-300, max_cycles=10,
                             cycles_per_launch=1, fused_pre=fused)
        with M.Multigrid(shape, hfm._lib.OP_SIGMA7, cfg, slots=1) as h:
            h.set_operator(hfm.ops.Sigma7(*(dev(T, sig[k]) for k in range(3))))
            h.load(0, dev(T, f))
            h.run(2)
            outs.append(h.fetch(0).cpu().numpy())
    close(outs[0], outs[1], rtol={"f32": 1e-5, "bf16": 2e-2, "f16": 3e-3}[storage])


def test_sawtooth_aspect_ratio_coarsest(hfm, T):
    """INHALE_demo.ipynb: flat domains (nz << nx, ny) coarsen to a 1 x r x r coarsest level
    (INH:13419); here 16 x 64 x 64 -> 1 x 4 x 4 with the NS pressure cycle (27-point w5, no
    fine-level Jacobi on w, x = X-1 rule), against the oracle."""
    b = np.zeros((16, 64, 64), np.float32)
    b[4:12, 20:40, 24:44] = 1.0
    b -= b.mean()
    ops = mg.hierarchy(mg.Stencil27(W.w5_pressure27()), 5)
    ref = np.zeros_like(b)
    for _ in range(2):
        ref = mg.sawtooth_cycle(ops, ref, b, fine_smooth=False, zero_xend=True)
    outs, levels = run_sawtooth(hfm, T, W.w5_pressure27(), b, np.zeros_like(b), 5, 2,
                                fine_smooth=False, zero_xend=True)
    assert levels[-1] == (1, 4, 4)
    close(outs[-1], ref)


@pytest.mark.parametrize("form", ["k27", "const7"])
def test_fused_coarse_cycle_other_operators(hfm, T, form):
    """The fused coarse V-cycle with the 27-point pressure kernel and the constant 7-point
    operator: F-cycles (whose V parts use it) agree with the separate-kernel path."""
    n = 32
    rng = np.random.default_rng(12)
    f = rng.standard_normal((n, n, n)).astype(np.float32)
    M, ops, L = hfm.multigrid, hfm.ops, hfm._lib
    if form == "k27":
        kind, op = L.OP_K27, ops.Stencil27(W.w5_pressure27())
    else:
        kind, op = L.OP_CONST7, ops.Const7(50.0, 100.0, 200.0)
    outs = []
    for fused in (True, False):
        cfg = M.SolverConfig(cycle="F", tol=1e-300, max_cycles=10, cycles_per_launch=1,
                             fused_coarse=fused)
        with M.Multigrid((n, n, n), kind, cfg, slots=8) as h:  # >= 8: the fused path runs
            h.set_operator(op)
            for s in range(8):
                h.load(s, dev(T, f))
            h.run(3)
            outs.append(h.fetch(5).cpu().numpy())
    close(outs[0], outs[1], rtol=1e-5)
