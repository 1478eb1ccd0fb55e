"""Two Jacobi sweeps per pass on FACE7 levels (temporal blocking) against one sweep per pass.

hfm_face7_smooth2_typed equals the two one-sweep entry points called in turn, bit for bit,
with and without the coarse correction, on grids with partial tiles and several z chunks:
tiles 64 wide (X <= 64), 128 wide (64 < X <= 128, one tile per row) and 64 wide with the
first sweep's ring columns computed cell by cell inside the grid (X > 128).

The two-sweep kernel recomputes the first sweep on a one-cell ring around its tile, in the
operation order of the tiles that own those cells, and stores it rounded to the storage type
as the one-sweep launches do.  Stationary V-cycles of a 16-bit handle therefore give the same
bits with and without HFM_OPT_TEMPORAL: the post-sweep pair (coarse correction, sweep,
sweep) on every FACE7 level and the pre-sweep pair (the fused first two sweeps from zero,
residual, restriction) on the zero-guess coarse FACE7 levels.  Grids cover partial tiles in
x (X = 48, X = 112) and y (Y = 24), several z chunks and several slots.

Float64 refinement around 16-bit PCG runs both pairs on the fine level, the last sweep
summing r . z; the partial sums there are grouped by the kernel's own blocks, so the
iterates agree to the refinement tolerance rather than bitwise: same status, iteration
counts within 2, true residual (float64 oracle operator) below 1e-6.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import mg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T(hfm):
    import torch
    return torch


def _problem(hfm, shape, B, seed, log_std=1.0):
    sig = np.stack([hfm.problems.anisotropic_sigma(shape, seed=seed + i, log_std=log_std)
                    for i in range(B)], axis=1)
    f = np.stack([hfm.problems.dipole(shape, seed=seed + i) for i in range(B)])
    return sig, f


def _face_op(hfm, T, dtype, sig, B, Z, Y, X):
    """FACE7 operator of conductivities sig (3, B, Z, Y, X), faces in the storage type."""
    L = hfm._lib
    code = {"bf16": L.BF16, "f16": L.F16}[dtype]
    tdt = {"bf16": T.bfloat16, "f16": T.float16}[dtype]
    fx = T.empty((B, Z, Y, X + 8), dtype=tdt, device="cuda")
    fy = T.empty((B, Z, Y + 1, X), dtype=tdt, device="cuda")
    fz = T.empty((B, Z + 1, Y, X), dtype=tdt, device="cuda")
    s = [T.from_numpy(np.ascontiguousarray(sig[k])).cuda() for k in range(3)]
    L.call("hfm_sigma7_faces", code, *(C.c_void_p(t.data_ptr()) for t in s), 0.5, 1.0, 2.0,
           *(C.c_void_p(t.data_ptr()) for t in (fx, fy, fz)), B, Z, Y, X, hfm.ops._stream())
    st = L.HfmOperator()
    st.kind, st.coef_dtype, st.scale = L.OP_FACE7, code, 1.0
    for i, t in enumerate((fx, fy, fz)):
        st.coef[i] = t.data_ptr()
    return st, (fx, fy, fz), code, tdt


@pytest.mark.parametrize("dtype", ["bf16", "f16"])
@pytest.mark.parametrize("shape,corr", [((2, 10, 20, 72), False), ((1, 12, 34, 128), True),
                                        ((3, 6, 16, 64), True), ((2, 4, 16, 48), True),
                                        ((1, 40, 48, 112), True), ((1, 6, 16, 192), True),
                                        ((2, 8, 24, 136), False)])
def test_smooth2_entry_point_equals_two_sweeps(hfm, T, dtype, shape, corr):
    """hfm_face7_smooth2_typed against hfm_prolong_correct_smooth_typed (or
    hfm_op_jacobi_typed) followed by hfm_op_jacobi_typed: the same bits."""
    L = hfm._lib
    B, Z, Y, X = shape
    rng = np.random.default_rng(sum(shape))
    sig = np.exp(rng.standard_normal((3,) + shape)).astype(np.float32)
    st, keep, code, tdt = _face_op(hfm, T, dtype, sig, B, Z, Y, X)
    rnd = lambda a: T.from_numpy(np.ascontiguousarray(a, np.float32)).cuda().to(tdt)
    phi = rnd(rng.standard_normal(shape))
    b = rnd(rng.standard_normal(shape))
    w = rnd(rng.standard_normal((B, Z // 2, Y // 2, X // 2))) if corr else None
    P = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None
    stream = hfm.ops._stream()
    om = 2.0 / 3.0
    out2 = T.empty_like(phi)
    L.call("hfm_face7_smooth2_typed", C.byref(st), code, P(phi), P(w), P(b), P(out2), B, Z, Y, X,
           om, stream)
    mid, out1 = T.empty_like(phi), T.empty_like(phi)
    if corr:
        L.call("hfm_prolong_correct_smooth_typed", C.byref(st), code, P(phi), P(w), P(b), P(mid),
               B, Z, Y, X, om, 0, stream)
    else:
        L.call("hfm_op_jacobi_typed", C.byref(st), code, P(phi), P(b), P(mid), B, Z, Y, X, om, 0,
               stream)
    L.call("hfm_op_jacobi_typed", C.byref(st), code, P(mid), P(b), P(out1), B, Z, Y, X, om, 0, stream)
    T.cuda.synchronize()
    a, r = out2.float().cpu().numpy(), out1.float().cpu().numpy()
    assert np.isfinite(a).all()
    np.testing.assert_array_equal(a, r)


def _op(hfm, T, sig):
    return hfm.ops.Sigma7(*(T.from_numpy(np.ascontiguousarray(sig[k])).cuda() for k in range(3)))


@pytest.mark.parametrize("storage", ["bf16", "f16"])
@pytest.mark.parametrize("shape,B", [((96, 96, 96), 2), ((80, 48, 224), 1), ((40, 24, 48), 3),
                                     ((64, 64, 112), 2)])
def test_stationary_vcycles_same_bits(hfm, T, storage, shape, B):
    M, L = hfm.multigrid, hfm._lib
    sig, f = _problem(hfm, shape, B, 70)
    outs = {}
    for temporal in (True, False):
        cfg = M.SolverConfig(cycle="V", storage=storage, tol=1e-300, max_cycles=10,
                             cycles_per_launch=1, temporal=temporal)
        with M.Multigrid(shape, L.OP_SIGMA7, cfg, slots=B) as h:
            h.set_operator(_op(hfm, T, sig))
            for s in range(B):
                h.load(s, T.from_numpy(f[s]).cuda())
            h.run(3)
            outs[temporal] = [h.fetch(s).cpu().numpy() for s in range(B)]
    for s in range(B):
        assert np.isfinite(outs[True][s]).all()
        np.testing.assert_array_equal(outs[True][s], outs[False][s])


@pytest.mark.parametrize("storage", ["bf16", "f16"])
@pytest.mark.parametrize("shape,B", [((64, 64, 64), 4), ((40, 24, 48), 2), ((96, 48, 112), 1)])
def test_refinement_agrees_with_one_sweep_per_pass(hfm, T, storage, shape, B):
    M, L = hfm.multigrid, hfm._lib
    sig, f = _problem(hfm, shape, B, 80, log_std=1.5)
    res = {}
    for temporal in (True, False):
        cfg = M.SolverConfig(cycle="V", accel="ir", storage=storage, tol=1e-6, max_cycles=600,
                             inner_tol=1e-3, temporal=temporal)
        with M.Multigrid(shape, L.OP_SIGMA7, cfg, slots=B) as h:
            h.set_operator(_op(hfm, T, sig))
            for s in range(B):
                h.load(s, T.from_numpy(f[s]).cuda())
            for _ in range(300):
                h.run(4)
                st = h.query()
                if not any(x["active"] for x in st):
                    break
            res[temporal] = ([h.fetch_f64(s).cpu().numpy() for s in range(B)], st)
    for s in range(B):
        x, st = res[True][0][s], res[True][1][s]
        st0 = res[False][1][s]
        assert st["status"] == 0 and st0["status"] == 0, (st, st0)
        assert abs(st["cycles"] - st0["cycles"]) <= 2, (st, st0)
        op64 = mg.Sigma7(sig[0, s], sig[1, s], sig[2, s], dtype=np.float64)
        assert mg.rel_residual(op64, x, f[s]) < 1e-6
        scale = np.abs(res[False][0][s]).max()
        assert np.abs(x - res[False][0][s]).max() <= 1e-4 * scale
