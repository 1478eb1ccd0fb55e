"""2D path on the GPU: the reference's Conv2D multigrid operators and cycle, the periodic
pressure V-cycle in float32 and bf16 storage, and the Kolmogorov-flow stepper, against the
oracle (``oracle/kolmogorov.py``).

Tolerances: float32 kernels vs the float32 oracle 1e-5 of the field's magnitude; float32
solves vs the float64 oracle 1e-4; bf16 storage one bf16 ulp (2^-8) of the magnitude.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import kolmogorov as K2, weights as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T(hfm):
    import torch
    return torch


def close(got, ref, rtol):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    err = np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-30)
    assert err <= rtol, "max rel err %.3e > %.1e" % (err, rtol)


def _w9(w):
    return (C.c_float * 9)(*[float(v) for v in np.asarray(w, np.float64).reshape(9)])


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("shape", [(1, 17, 23), (3, 64, 48)])
def test_conv_restrict_prolong(hfm, T, periodic, shape):
    L, ops = hfm._lib, hfm.ops
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape).astype(np.float32)
    w = rng.standard_normal((3, 3)).astype(np.float32)
    xd = T.from_numpy(x).cuda()
    y = T.empty_like(xd)
    flags = L.FLAG_PERIODIC if periodic else 0
    B, Y, X = shape
    L.call("hfm_conv2d_k3", C.c_void_p(xd.data_ptr()), C.c_void_p(y.data_ptr()), B, Y, X, _w9(w),
           flags, ops._stream())
    ref = np.stack([K2.conv2d(x[i], w, periodic) for i in range(B)])
    close(y.cpu().numpy(), ref, 1e-5)
    c = T.empty((B, Y // 2, X // 2), device="cuda")
    L.call("hfm_restrict_avg2d", L.F32, C.c_void_p(xd.data_ptr()), C.c_void_p(c.data_ptr()), B, Y, X,
           ops._stream())
    close(c.cpu().numpy(), np.stack([K2.restrict2d(x[i]) for i in range(B)]), 1e-6)
    f = T.empty((B, 2 * (Y // 2), 2 * (X // 2)), device="cuda")
    L.call("hfm_prolong_nearest2d", L.F32, C.c_void_p(c.data_ptr()), C.c_void_p(f.data_ptr()), B,
           Y // 2, X // 2, ops._stream())
    np.testing.assert_array_equal(f.cpu().numpy(), np.stack([K2.prolong2d(K2.restrict2d(x[i])) for i in range(B)]))


@pytest.mark.parametrize("storage", ["f32", "bf16"])
@pytest.mark.parametrize("periodic", [False, True])
def test_jacobi_and_residual_restrict(hfm, T, storage, periodic):
    L, ops = hfm._lib, hfm.ops
    code, tdt = {"f32": (L.F32, T.float32), "bf16": (L.BF16, T.bfloat16)}[storage]
    rng = np.random.default_rng(2)
    B, Y, X = 2, 32, 40
    phi = T.from_numpy(rng.standard_normal((B, Y, X)).astype(np.float32)).cuda().to(tdt)
    rhs = T.from_numpy(rng.standard_normal((B, Y, X)).astype(np.float32)).cuda().to(tdt)
    wc = T.from_numpy(rng.standard_normal((B, Y // 2, X // 2)).astype(np.float32)).cuda().to(tdt)
    w = K2.laplace5(1.0)
    flags = L.FLAG_PERIODIC if periodic else 0
    out = T.empty_like(phi)
    L.call("hfm_jacobi2d", code, _w9(w), C.c_void_p(phi.data_ptr()), C.c_void_p(wc.data_ptr()), -1.0,
           C.c_void_p(rhs.data_ptr()), C.c_void_p(out.data_ptr()), B, Y, X, 0.8, flags, ops._stream())
    p64, r64, c64 = (t.double().cpu().numpy() for t in (phi, rhs, wc))
    ref = np.stack([K2.jacobi2d(w, p64[i] - K2.prolong2d(c64[i]), r64[i], 0.8, periodic, np.float64)
                    for i in range(B)])
    close(out.double().cpu().numpy(), ref, 1e-5 if storage == "f32" else 2 ** -8)
    rc = T.empty((B, Y // 2, X // 2), dtype=tdt, device="cuda")
    L.call("hfm_residual_restrict2d", code, _w9(w), C.c_void_p(phi.data_ptr()), C.c_void_p(rhs.data_ptr()),
           C.c_void_p(rc.data_ptr()), B, Y, X, flags, ops._stream())
    ref = np.stack([K2.restrict2d(K2.conv2d(p64[i], w, periodic, np.float64) - r64[i]) for i in range(B)])
    close(rc.double().cpu().numpy(), ref, 1e-5 if storage == "f32" else 2 ** -8)


def test_reference_2d_cycle_matches_oracle(hfm, T):
    """Three cycles of Multigrid_2D.ipynb#c18 on its own problem (128^2, the cell-3 weights,
    a 40 x 40 box source at (43, 43), initial guess = the source)."""
    KM = hfm.kolmogorov
    w = hfm.weights.advection_diffusion_2d()
    b = np.zeros((128, 128), np.float32)
    b[43:83, 43:83] = 1.0
    mg = KM.Multigrid2D((128, 128), w, storage="f32", periodic=False, coarse_scale=1.0,
                        min_edge=1, omega=1.0)
    bd = T.from_numpy(b).cuda().view(1, 128, 128)
    v = bd.clone()
    ref = b.copy()
    nl = len(K2.level_shapes((128, 128), 1))
    assert mg.L == nl
    for _ in range(3):
        v = mg.sawtooth(v, bd)
        ref = K2.sawtooth2d(W.w2_2d_advection_diffusion(), ref, b, nl)
    close(v[0].cpu().numpy(), ref, 1e-5)


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_periodic_pressure_cycles(hfm, T, storage):
    """Outer iterations p -= V(A p - f) on the periodic 5-point Poisson problem agree with the
    float64 oracle (float32 storage) and converge to the storage's limit (bf16)."""
    KM = hfm.kolmogorov
    n = 64
    h = 2 * np.pi / n
    rng = np.random.default_rng(4)
    f = rng.standard_normal((n, n))
    f -= f.mean()
    mg = KM.Multigrid2D((n, n), KM.laplace5(h), storage=storage)
    om = K2.VCycle2D(K2.laplace5(h), (n, n))
    fd = T.from_numpy(f.astype(np.float32)).cuda().view(1, n, n)
    p = T.zeros((1, n, n), device="cuda")
    mg.solve(p, fd, 3)
    ref = om.solve(np.zeros((n, n)), f, 3)
    close(p[0].cpu().numpy(), ref, 1e-4 if storage == "f32" else 2e-2)
    mg.solve(p, fd, 5)
    res = mg.rel_residual(p, fd)[0]
    assert res < (1e-5 if storage == "f32" else 2e-3), res
    assert abs(float(p.double().mean())) < 1e-6


@pytest.mark.parametrize("storage", ["f32", "bf16"])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("shape", [(1, 17, 23), (3, 64, 48), (2, 512, 512)])
def test_two_sweeps_from_zero_same_bits(hfm, T, storage, periodic, shape):
    """hfm_jacobi2d with HFM_FLAG_TWO_SWEEPS equals two hfm_jacobi2d calls from zero, bit for
    bit, in float32 and bf16 storage (the first sweep rounded to the storage type)."""
    L = hfm._lib
    KM = hfm.kolmogorov
    code, tdt = KM._DT[storage]
    rng = np.random.default_rng(sum(shape))
    w = rng.standard_normal((3, 3))
    w[1, 1] = 2.0 + np.abs(w).sum()
    f = T.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda().to(tdt)
    B, Y, X = shape
    fl = L.FLAG_PERIODIC if periodic else 0
    P = lambda t: C.c_void_p(t.data_ptr())
    st = hfm.ops._stream()
    one, two, fused = T.empty_like(f), T.empty_like(f), T.empty_like(f)
    L.call("hfm_jacobi2d", code, _w9(w), None, None, 0.0, P(f), P(one), B, Y, X, 0.8, fl, st)
    L.call("hfm_jacobi2d", code, _w9(w), P(one), None, 0.0, P(f), P(two), B, Y, X, 0.8, fl, st)
    L.call("hfm_jacobi2d", code, _w9(w), None, None, 0.0, P(f), P(fused), B, Y, X, 0.8,
           fl | L.FLAG_TWO_SWEEPS, st)
    T.cuda.synchronize()
    a, r = fused.float().cpu().numpy(), two.float().cpu().numpy()
    assert np.isfinite(a).all()
    np.testing.assert_array_equal(a, r)


@pytest.mark.parametrize("storage", ["f32", "bf16"])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("shape", [(17, 23), (1, 9), (40, 72)])
def test_two_sweeps_with_correction_same_bits(hfm, T, storage, periodic, shape):
    """hfm_jacobi2d with HFM_FLAG_TWO_SWEEPS from base - P(coarse) (or base alone) equals the
    correction + sweep launch followed by a plain sweep, bit for bit; partial tiles in x and
    y and a one-row grid."""
    L = hfm._lib
    KM = hfm.kolmogorov
    code, tdt = KM._DT[storage]
    Y, X = shape
    corr = Y % 2 == 0 and X % 2 == 0
    B = 2
    rng = np.random.default_rng(Y * X)
    w = rng.standard_normal((3, 3))
    w[1, 1] = 2.0 + np.abs(w).sum()
    rnd = lambda s: T.from_numpy(rng.standard_normal(s).astype(np.float32)).cuda().to(tdt)
    f, base = rnd((B, Y, X)), rnd((B, Y, X))
    wc = rnd((B, Y // 2, X // 2)) if corr else None
    fl = L.FLAG_PERIODIC if periodic else 0
    P = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    st = hfm.ops._stream()
    one, two, fused = T.empty_like(f), T.empty_like(f), T.empty_like(f)
    L.call("hfm_jacobi2d", code, _w9(w), P(base), P(wc), -1.0, P(f), P(one), B, Y, X, 0.8, fl, st)
    L.call("hfm_jacobi2d", code, _w9(w), P(one), None, 0.0, P(f), P(two), B, Y, X, 0.8, fl, st)
    L.call("hfm_jacobi2d", code, _w9(w), P(base), P(wc), -1.0, P(f), P(fused), B, Y, X, 0.8,
           fl | L.FLAG_TWO_SWEEPS, st)
    T.cuda.synchronize()
    a, r = fused.float().cpu().numpy(), two.float().cpu().numpy()
    assert np.isfinite(a).all()
    np.testing.assert_array_equal(a, r)


@pytest.mark.parametrize("storage", ["f32", "bf16"])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("shape", [(1, 18, 44), (2, 2, 2), (3, 64, 48), (1, 512, 512)])
def test_pre2_restrict_same_bits(hfm, T, storage, periodic, shape):
    """hfm_pre2_restrict2d equals hfm_jacobi2d (two sweeps from zero) followed by
    hfm_residual_restrict2d, bit for bit: the iterate and the coarse rhs; partial tiles and a
    2 x 2 grid."""
    L = hfm._lib
    KM = hfm.kolmogorov
    code, tdt = KM._DT[storage]
    B, Y, X = shape
    rng = np.random.default_rng(Y + X + B)
    w = rng.standard_normal((3, 3))
    w[1, 1] = 2.0 + np.abs(w).sum()
    f = T.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda().to(tdt)
    fl = L.FLAG_PERIODIC if periodic else 0
    P = lambda t: C.c_void_p(t.data_ptr())
    st = hfm.ops._stream()
    phi_r, phi_f = T.empty_like(f), T.empty_like(f)
    fc_r = T.empty((B, Y // 2, X // 2), dtype=tdt, device="cuda")
    fc_f = T.empty_like(fc_r)
    L.call("hfm_jacobi2d", code, _w9(w), None, None, 0.0, P(f), P(phi_r), B, Y, X, 0.8,
           fl | L.FLAG_TWO_SWEEPS, st)
    L.call("hfm_residual_restrict2d", code, _w9(w), P(phi_r), P(f), P(fc_r), B, Y, X, fl, st)
    L.call("hfm_pre2_restrict2d", code, _w9(w), P(f), P(phi_f), P(fc_f), B, Y, X, 0.8, fl, st)
    T.cuda.synchronize()
    for a, r in ((phi_f, phi_r), (fc_f, fc_r)):
        a, r = a.float().cpu().numpy(), r.float().cpu().numpy()
        assert np.isfinite(a).all()
        np.testing.assert_array_equal(a, r)


@pytest.mark.parametrize("storage", ["f32", "bf16"])
@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("nu", [(2, 2), (3, 3)])
def test_fused_pairs_cycle_same_bits(hfm, T, storage, periodic, nu):
    """Outer iterations with and without the fused pairs of sweeps: the same bits."""
    KM = hfm.kolmogorov
    Y, X, slots = 256, 192, 2
    rng = np.random.default_rng(7)
    w = KM.laplace5(2 * np.pi / X)
    if not periodic:
        w[1, 1] *= 1.1
    f = rng.standard_normal((slots, Y, X)).astype(np.float32)
    f -= f.mean(axis=(1, 2), keepdims=True)
    fd = T.from_numpy(f).cuda()
    out = {}
    for fused in (True, False):
        mg = KM.Multigrid2D((Y, X), w, storage=storage, periodic=periodic, nu_pre=nu[0],
                            nu_post=nu[1], slots=slots, fused_pairs=fused)
        p = T.zeros((slots, Y, X), device="cuda")
        for _ in range(3):
            mg.iterate(p, fd)
        out[fused] = p.cpu().numpy()
    assert np.isfinite(out[True]).all()
    np.testing.assert_array_equal(out[True], out[False])


@pytest.mark.parametrize("periodic", [True, False])
@pytest.mark.parametrize("shape,slots,nu", [((512, 512), 1, (2, 2)), ((64, 64), 2, (2, 2)),
                                            ((128, 96), 3, (1, 0)), ((256, 64), 1, (3, 1))])
def test_fused_coarse_cycle_same_bits(hfm, T, periodic, shape, slots, nu):
    """Outer iterations with the levels of at most 4096 cells in one launch (hfm_subcycle2d)
    give the bits of the per-level launches in float32 storage, and agree to bf16 rounding in
    bf16 storage (the fused launch keeps those levels in float32)."""
    KM = hfm.kolmogorov
    Y, X = shape
    rng = np.random.default_rng(Y + X + slots)
    w = KM.laplace5(2 * np.pi / X)
    if not periodic:
        w[1, 1] *= 1.1  # diagonally dominant
    f = rng.standard_normal((slots, Y, X)).astype(np.float32)
    if periodic:
        f -= f.mean(axis=(1, 2), keepdims=True)
    fd = T.from_numpy(f).cuda()
    out = {}
    for storage in ("f32", "bf16"):
        for fused in (True, False):
            mg = KM.Multigrid2D(shape, w, storage=storage, periodic=periodic, nu_pre=nu[0],
                                nu_post=nu[1], slots=slots, fused_coarse=fused)
            assert mg.fused_coarse == fused
            p = T.zeros((slots, Y, X), device="cuda")
            for _ in range(3):
                mg.iterate(p, fd)
            out[storage, fused] = p.cpu().numpy()
    assert np.isfinite(out["f32", True]).all()
    np.testing.assert_array_equal(out["f32", True], out["f32", False])
    close(out["bf16", True], out["f32", False], 2e-2)
    close(out["bf16", True], out["bf16", False], 2e-2)


def test_kolmogorov_step_matches_oracle(hfm, T):
    KM = hfm.kolmogorov
    n = 64
    kf = KM.KolmogorovFlow(n=n, dt=2e-3, cycles=3, seed=5)
    u0, v0, p0 = (t.double().cpu().numpy() for t in (kf.u, kf.v, kf.p))
    om = K2.VCycle2D(K2.laplace5(kf.h), (n, n), dt=np.float64)
    kf.step()
    u1, v1, p1 = K2.ns_step(u0, v0, p0, om, 3, kf.dt, kf.nu, kf.h)
    close(kf.u.cpu().numpy(), u1, 1e-5)
    close(kf.v.cpu().numpy(), v1, 1e-4)
    close(kf.p.cpu().numpy(), p1, 1e-3)


def test_kolmogorov_graph_replay_equals_eager(hfm, T):
    KM = hfm.kolmogorov
    a = KM.KolmogorovFlow(n=64, dt=2e-3, seed=6)
    b = KM.KolmogorovFlow(n=64, dt=2e-3, seed=6)
    a.run(46, per_graph=20)   # 2 set-up steps + 2 replays + 4 eager steps
    for _ in range(46):
        b.step()
    T.cuda.synchronize()
    assert a.steps_done == b.steps_done == 46
    np.testing.assert_array_equal(a.u.cpu().numpy(), b.u.cpu().numpy())
    np.testing.assert_array_equal(a.p.cpu().numpy(), b.p.cpu().numpy())
    d = a.diagnostics()
    assert np.isfinite(d["energy"]) and d["max_abs_div"] < 1e-2 * d["max_u"] / a.h


def test_kolmogorov_bf16_pressure_tracks_f32(hfm, T):
    KM = hfm.kolmogorov
    runs = {}
    for st in ("f32", "bf16"):
        kf = KM.KolmogorovFlow(n=128, dt=1e-3, storage=st, seed=7)
        kf.run(200, per_graph=50)
        runs[st] = kf.diagnostics()
    e32, e16 = runs["f32"]["energy"], runs["bf16"]["energy"]
    assert abs(e32 - e16) / e32 < 1e-3, (e32, e16)
    assert runs["bf16"]["pressure_rel_resid"] < 0.05
