"""The face-coefficient operator (FACE7) on the GPU against the oracle.

hfm_sigma7_faces forms the SIGMA7 faces in float32 and rounds each once to the storage type;
the oracle (``mg.sigma7_faces``) does the same, so the face arrays agree bit for bit.  The
16-bit FACE7 kernels (plane-marching with mixed-precision FMAs on the TMA-eligible grids, the
generic kernels elsewhere) are then compared with the float64 oracle operator built from
those rounded faces and the rounded fields: one unit of the storage type's last place of
each result plus the float32 evaluation error (1e-5 of the operands' scale).  Handle tests
check that V-cycles and solves with faces agree with the conductivity path and the float32
handle to the storage precision and reach their tolerance.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import mg, tfops

pytestmark = pytest.mark.gpu

ULP = {"bf16": 2.0 ** -8, "f16": 2.0 ** -11}
CC = (0.5, 1.0, 2.0)
# (B, Z, Y, X): TMA-eligible grids (X >= 48, Y >= 16, partial tiles in x and y, X = 48), and
# grids the generic kernels take (Y < 16, X not a multiple of 8)
SHAPES = [(2, 10, 20, 72), (1, 12, 34, 128), (3, 6, 16, 64), (2, 4, 16, 48), (2, 6, 10, 40),
          (2, 6, 8, 6)]


@pytest.fixture(scope="module")
def T(hfm):
    import torch
    return torch


def _tdt(T, dtype):
    return {"f32": T.float32, "bf16": T.bfloat16, "f16": T.float16}[dtype]


def _faces(hfm, T, dtype, sig, B, Z, Y, X):
    L = hfm._lib
    code = {"f32": L.F32, "bf16": L.BF16, "f16": L.F16}[dtype]
    nfx, nfy, nfz = C.c_int64(), C.c_int64(), C.c_int64()
    L.call("hfm_face7_elems", Z, Y, X, C.byref(nfx), C.byref(nfy), C.byref(nfz))
    assert (nfx.value, nfy.value, nfz.value) == (Z * Y * (X + 8), Z * (Y + 1) * X, (Z + 1) * Y * X)
    tdt = _tdt(T, dtype)
    fx = T.empty((B, Z, Y, X + 8), dtype=tdt, device="cuda")
    fy = T.empty((B, Z, Y + 1, X), dtype=tdt, device="cuda")
    fz = T.empty((B, Z + 1, Y, X), dtype=tdt, device="cuda")
    s = [T.from_numpy(np.ascontiguousarray(sig[k])).cuda() for k in range(3)]
    L.call("hfm_sigma7_faces", code, *(C.c_void_p(t.data_ptr()) for t in s), *CC,
           *(C.c_void_p(t.data_ptr()) for t in (fx, fy, fz)), B, Z, Y, X, hfm.ops._stream())
    T.cuda.synchronize()
    return fx, fy, fz


@pytest.mark.parametrize("dtype", ["f32", "bf16", "f16"])
def test_sigma7_faces_match_oracle_bitwise(hfm, T, dtype):
    B, Z, Y, X = 2, 5, 7, 24
    rng = np.random.default_rng(3)
    sig = np.exp(2 * rng.standard_normal((3, B, Z, Y, X))).astype(np.float32)
    got = _faces(hfm, T, dtype, sig, B, Z, Y, X)
    ref = mg.sigma7_faces(sig[0], sig[1], sig[2], c=CC, storage=dtype)
    for g, r in zip(got, ref):
        np.testing.assert_array_equal(g.float().cpu().numpy(), r)


def _setup(hfm, T, dtype, shape, seed):
    L = hfm._lib
    B, Z, Y, X = shape
    rng = np.random.default_rng(seed)
    sig = np.exp(rng.standard_normal((3,) + shape)).astype(np.float32)
    tdt = _tdt(T, dtype)
    rnd = lambda a: T.from_numpy(np.ascontiguousarray(a, np.float32)).cuda().to(tdt)
    x = rnd(rng.standard_normal(shape))
    b = rnd(rng.standard_normal(shape))
    fx, fy, fz = _faces(hfm, T, dtype, sig, B, Z, Y, X)
    st = L.HfmOperator()
    st.kind = L.OP_FACE7
    st.coef_dtype = {"bf16": L.BF16, "f16": L.F16}[dtype]
    st.scale = 1.0
    for k, t in enumerate((fx, fy, fz)):
        st.coef[k] = t.data_ptr()
    ops = [mg.Face7(fx[i].double().cpu().numpy(), fy[i].double().cpu().numpy(),
                    fz[i].double().cpu().numpy()) for i in range(B)]
    keep = (fx, fy, fz)
    return st, ops, x, b, keep


def _check(got, ref, dtype, scale):
    excess = np.abs(got - ref) - ULP[dtype] * np.abs(ref)
    assert excess.max() <= 1e-5 * scale, excess.max() / scale


@pytest.mark.parametrize("dtype", ["bf16", "f16"])
@pytest.mark.parametrize("shape", SHAPES)
def test_face7_jacobi_and_residual(hfm, T, dtype, shape):
    L = hfm._lib
    B, Z, Y, X = shape
    st, ops, x, b, keep = _setup(hfm, T, dtype, shape, 11)
    code = st.coef_dtype
    P = lambda t: C.c_void_p(t.data_ptr())
    stream = hfm.ops._stream()
    x64, b64 = x.double().cpu().numpy(), b.double().cpu().numpy()
    out = T.empty_like(x)
    L.call("hfm_op_jacobi_typed", C.byref(st), code, P(x), P(b), P(out), B, Z, Y, X, 0.8, 0, stream)
    ref = np.stack([mg.jacobi(ops[i], x64[i], b64[i], 0.8) for i in range(B)])
    dmax = max(float(op.diag.max()) for op in ops)
    _check(out.double().cpu().numpy(), ref, dtype, max(np.abs(ref).max(), np.abs(x64).max(), np.abs(b64).max()))
    # zero initial guess: phi is not read
    L.call("hfm_op_jacobi_typed", C.byref(st), code, None, P(b), P(out), B, Z, Y, X, 0.8,
           L.FLAG_ZERO_GUESS, stream)
    ref = np.stack([mg.jacobi(ops[i], np.zeros_like(b64[i]), b64[i], 0.8) for i in range(B)])
    _check(out.double().cpu().numpy(), ref, dtype, max(np.abs(ref).max(), np.abs(b64).max()))
    L.call("hfm_op_residual_typed", C.byref(st), code, P(x), P(b), P(out), B, Z, Y, X, 0, stream)
    ref = np.stack([mg.residual(ops[i], x64[i], b64[i]) for i in range(B)])
    _check(out.double().cpu().numpy(), ref, dtype, dmax * np.abs(x64).max() + np.abs(b64).max())


@pytest.mark.parametrize("dtype", ["bf16", "f16"])
@pytest.mark.parametrize("shape", [s for s in SHAPES if not any(v & 1 for v in s[1:])])
def test_face7_fused_transfers(hfm, T, dtype, shape):
    """Residual + restriction and prolongation + correction + sweep (both signs of the
    correction: phi - P w of the V-cycle, and P w alone of the sawtooth)."""
    L = hfm._lib
    B, Z, Y, X = shape
    st, ops, x, b, keep = _setup(hfm, T, dtype, shape, 13)
    code = st.coef_dtype
    P = lambda t: C.c_void_p(t.data_ptr())
    stream = hfm.ops._stream()
    x64, b64 = x.double().cpu().numpy(), b.double().cpu().numpy()
    dmax = max(float(op.diag.max()) for op in ops)
    rc = T.empty((B, Z // 2, Y // 2, X // 2), dtype=x.dtype, device="cuda")
    rf = T.empty_like(x)
    L.call("hfm_residual_restrict_typed", C.byref(st), code, P(x), P(b), P(rf), P(rc), B, Z, Y, X,
           0, stream)
    r = np.stack([mg.residual(ops[i], x64[i], b64[i]) for i in range(B)])
    scale = dmax * np.abs(x64).max() + np.abs(b64).max()
    _check(rf.double().cpu().numpy(), r, dtype, scale)
    _check(rc.double().cpu().numpy(), tfops.restrict_avg(r, np.float64), dtype, scale)
    rng = np.random.default_rng(5)
    wc = T.from_numpy(rng.standard_normal((B, Z // 2, Y // 2, X // 2)).astype(np.float32)).cuda().to(x.dtype)
    w64 = wc.double().cpu().numpy()
    out = T.empty_like(x)
    L.call("hfm_prolong_correct_smooth_typed", C.byref(st), code, P(x), P(wc), P(b), P(out), B, Z,
           Y, X, 2.0 / 3.0, 0, stream)
    ref = np.stack([mg.jacobi(ops[i], x64[i] - tfops.prolong_nearest(w64[i], np.float64), b64[i],
                              2.0 / 3.0) for i in range(B)])
    _check(out.double().cpu().numpy(), ref, dtype, max(np.abs(ref).max(), np.abs(x64).max(), np.abs(w64).max()))
    L.call("hfm_prolong_correct_smooth_typed", C.byref(st), code, None, P(wc), P(b), P(out), B, Z,
           Y, X, 1.0, 0, stream)
    ref = np.stack([mg.jacobi(ops[i], tfops.prolong_nearest(w64[i], np.float64), b64[i], 1.0)
                    for i in range(B)])
    _check(out.double().cpu().numpy(), ref, dtype, max(np.abs(ref).max(), np.abs(w64).max()))


def test_face7_scale_multiplies_the_operator(hfm, T):
    L = hfm._lib
    shape = (2, 6, 16, 64)
    B, Z, Y, X = shape
    st, ops, x, b, keep = _setup(hfm, T, "bf16", shape, 17)
    st.scale = 0.25
    P = lambda t: C.c_void_p(t.data_ptr())
    out = T.empty_like(x)
    L.call("hfm_op_residual_typed", C.byref(st), st.coef_dtype, P(x), P(b), P(out), B, Z, Y, X, 0,
           hfm.ops._stream())
    x64, b64 = x.double().cpu().numpy(), b.double().cpu().numpy()
    ref = np.stack([0.25 * ops[i].apply(x64[i]) - b64[i] for i in range(B)])
    dmax = max(float(op.diag.max()) for op in ops)
    _check(out.double().cpu().numpy(), ref, "bf16", dmax * np.abs(x64).max() + np.abs(b64).max())


@pytest.mark.parametrize("storage", ["bf16", "f16"])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 48, 96)])
def test_vcycles_with_faces_agree_with_conductivity_path(hfm, T, storage, shape):
    """Stationary V-cycles of a 16-bit handle with faces on its TMA levels against the same
    handle without (HFM_OPT_NO_FACES) and the float32 handle: the storage precision."""
    sig = hfm.problems.anisotropic_sigma(shape, seed=4, log_std=1.0)
    f = hfm.problems.dipole(shape, seed=4)
    M = hfm.multigrid
    outs = {}
    for name, st, faces in (("f32", "f32", True), ("faces", storage, True), ("sigma", storage, False)):
        cfg = M.SolverConfig(cycle="V", storage=st, tol=1e-300, max_cycles=10, cycles_per_launch=1,
                             faces=faces)
        with M.Multigrid(shape, hfm._lib.OP_SIGMA7, cfg, slots=2) as h:
            for s in range(2):
                h.set_operator(hfm.ops.Sigma7(*(T.from_numpy(sig[k]).cuda() for k in range(3))), slot=s)
                h.load(s, T.from_numpy(f).cuda())
            h.run(2)
            outs[name] = [h.fetch(s).cpu().numpy() for s in range(2)]
    tol = 3e-2 if storage == "bf16" else 5e-3
    for s in range(2):
        ref = np.abs(outs["f32"][s]).max()
        assert np.abs(outs["faces"][s] - outs["f32"][s]).max() / ref < tol
        assert np.abs(outs["faces"][s] - outs["sigma"][s]).max() / ref < tol
    np.testing.assert_array_equal(outs["faces"][0], outs["faces"][1])


@pytest.mark.parametrize("storage", ["bf16", "f16"])
@pytest.mark.parametrize("n", [64, 128])
def test_refinement_with_faces_reaches_tolerance(hfm, T, storage, n):
    """float64 refinement around 16-bit inner cycles with faces: the true residual (float64
    oracle operator) reaches 1e-6 and the iteration count stays that of the conductivity
    path within 15 %."""
    M, L = hfm.multigrid, hfm._lib
    sig = hfm.problems.anisotropic_sigma((n, n, n), seed=8, log_std=1.5)
    f = hfm.problems.dipole((n, n, n), seed=8)
    res = {}
    for faces in (True, False):
        cfg = M.SolverConfig(cycle="V", accel="ir", storage=storage, tol=1e-6, max_cycles=600,
                             inner_tol=1e-3, faces=faces)
        with M.Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=1) as h:
            h.set_operator(hfm.ops.Sigma7(*(T.from_numpy(sig[k]).cuda() for k in range(3))))
            h.load(0, T.from_numpy(f).cuda())
            for _ in range(200):
                h.run(4)
                s = h.query()[0]
                if not s["active"]:
                    break
            res[faces] = (h.fetch_f64(0).cpu().numpy(), s)
    op64 = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float64)
    for faces, (x, s) in res.items():
        assert s["status"] == 0, (faces, s)
        assert mg.rel_residual(op64, x, f) < 1e-6
    c1, c0 = res[True][1]["cycles"], res[False][1]["cycles"]
    assert abs(c1 - c0) <= max(2, 0.15 * c0), (c1, c0)
