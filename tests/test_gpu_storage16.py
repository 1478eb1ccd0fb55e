"""16-bit storage kernels (bf16 / fp16 fields and conductivities, float32 arithmetic).

The typed Jacobi sweep is compared with the float64 oracle evaluated on the same rounded
inputs: the kernel computes in float32 and rounds its result once, so the bound is one unit
of the storage type's last place (2^-8 bf16, 2^-11 fp16, relative to each value) plus the
float32 evaluation error (1e-5 of the operands' scale).  Shapes cover the TMA kernels (X >= 64,
Y >= 16, partial tiles in x and y), the register-queue kernels (X % 4 == 0, X < 64), the
generic kernels, and views whose data pointer is not 16-byte aligned (the dispatch takes the
scalar kernels for those).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import mg, weights as W

pytestmark = pytest.mark.gpu

ULP = {"bf16": 2.0 ** -8, "f16": 2.0 ** -11}
SHAPES = [(2, 9, 20, 72), (1, 12, 33, 128), (3, 5, 16, 64), (2, 6, 10, 40), (2, 5, 7, 6)]


@pytest.fixture(scope="module")
def T(hfm):
    import torch
    return torch


def _round(T, a, tdt):
    """numpy float32 -> device tensor of the storage type, and its exact float64 value."""
    t = T.from_numpy(np.ascontiguousarray(a)).cuda().to(tdt)
    return t, t.double().cpu().numpy()


def _typed_jacobi(hfm, T, form, dtype, shape, omega, flags=0, offset=0, seed=0):
    L = hfm._lib
    tdt = {"bf16": T.bfloat16, "f16": T.float16}[dtype]
    code = {"bf16": L.BF16, "f16": L.F16}[dtype]
    rng = np.random.default_rng(seed)
    B = shape[0]
    x = rng.standard_normal(shape).astype(np.float32)
    b = rng.standard_normal(shape).astype(np.float32)
    xt, x64 = _round(T, x, tdt)
    bt, b64 = _round(T, b, tdt)
    if offset:
        # same values at a data pointer `offset` elements past an aligned allocation
        xs = T.empty(xt.numel() + offset, dtype=tdt, device="cuda")
        xs[offset:] = xt.reshape(-1)
        xt = xs[offset:].view(shape)
    out = T.empty(shape, dtype=tdt, device="cuda")
    st = L.HfmOperator()
    st.coef_dtype = code
    st.scale = 1.0
    keep = []
    if form == "sigma7":
        sig = np.exp(rng.standard_normal((3,) + shape)).astype(np.float32)
        s64 = []
        for k in range(3):
            t, v = _round(T, sig[k], tdt)
            keep.append(t)
            s64.append(v)
            st.coef[k] = t.data_ptr()
            st.c[k] = (0.5, 1.0, 2.0)[k]
        st.kind = L.OP_SIGMA7
        ops = [mg.Sigma7(s64[0][i], s64[1][i], s64[2][i], c=(0.5, 1.0, 2.0), dtype=np.float64)
               for i in range(B)]
    elif form == "const7":
        st.kind = L.OP_CONST7
        st.k[0], st.k[1], st.k[2] = 0.5, 1.0, 2.0
        ops = [mg.const7(0.5, 1.0, 2.0, dtype=np.float64)] * B
    else:
        K = W.w5_pressure27().astype(np.float32)
        st.kind = L.OP_K27
        for i, v in enumerate(K.reshape(27)):
            st.k[i] = float(v)
        ops = [mg.Stencil27(K.astype(np.float64), dtype=np.float64)] * B
    stream = hfm.ops._stream()
    L.call("hfm_op_jacobi_typed", C.byref(st), code, C.c_void_p(xt.data_ptr()),
           C.c_void_p(bt.data_ptr()), C.c_void_p(out.data_ptr()), B, shape[1], shape[2],
           shape[3], omega, flags, stream)
    T.cuda.synchronize()
    got = out.double().cpu().numpy()
    xin = np.zeros_like(x64) if flags & L.FLAG_ZERO_GUESS else x64.copy()
    if flags & L.FLAG_ZERO_XEND:
        xin[..., -1] = 0.0
    ref = np.stack([mg.jacobi(ops[i], xin[i], b64[i], omega) for i in range(B)])
    return got, ref, max(np.abs(x64).max(), np.abs(b64).max(), np.abs(ref).max())


@pytest.mark.parametrize("dtype", ["bf16", "f16"])
@pytest.mark.parametrize("form", ["sigma7", "const7", "k27"])
@pytest.mark.parametrize("shape", SHAPES)
def test_typed_jacobi_matches_oracle(hfm, T, dtype, form, shape):
    got, ref, scale = _typed_jacobi(hfm, T, form, dtype, shape, 2.0 / 3.0)
    excess = np.abs(got - ref) - ULP[dtype] * np.abs(ref)
    assert excess.max() <= 1e-5 * scale, excess.max() / scale


@pytest.mark.parametrize("dtype", ["bf16", "f16"])
def test_typed_jacobi_flags(hfm, T, dtype):
    L = hfm._lib
    for flags in (L.FLAG_ZERO_GUESS, L.FLAG_ZERO_XEND):
        got, ref, scale = _typed_jacobi(hfm, T, "sigma7", dtype, (2, 9, 20, 72), 0.8, flags=flags)
        excess = np.abs(got - ref) - ULP[dtype] * np.abs(ref)
        assert excess.max() <= 1e-5 * scale, (flags, excess.max() / scale)


@pytest.mark.parametrize("offset", [1, 2, 4])
def test_unaligned_views_take_scalar_kernels(hfm, T, offset):
    """A phi view 2 / 4 / 8 bytes past a 16-byte boundary gives the same result as the
    aligned call (the vector kernels are skipped for it)."""
    a, ref, _ = _typed_jacobi(hfm, T, "sigma7", "bf16", (2, 9, 20, 72), 2.0 / 3.0, seed=5)
    b, _, _ = _typed_jacobi(hfm, T, "sigma7", "bf16", (2, 9, 20, 72), 2.0 / 3.0, offset=offset,
                            seed=5)
    excess = np.abs(b - ref) - ULP["bf16"] * np.abs(ref)
    assert excess.max() <= 1e-5 * np.abs(ref).max()
    assert np.abs(a - b).max() <= 2 * ULP["bf16"] * np.abs(ref).max()


@pytest.mark.parametrize("storage", ["bf16", "f16"])
@pytest.mark.parametrize("shape", [(64, 64, 64), (24, 48, 80)])
def test_vcycle_16bit_storage_on_tma_levels(hfm, T, storage, shape):
    """V-cycles whose fine level runs the 16-bit TMA kernels (smoother, residual +
    restriction, prolongation + correction + smoothing) agree with the float32 handle to the
    storage precision."""
    sig = hfm.problems.anisotropic_sigma(shape, seed=3, log_std=1.0)
    f = hfm.problems.dipole(shape, seed=3)
    M = hfm.multigrid
    outs = {}
    for st in ("f32", storage):
        cfg = M.SolverConfig(cycle="V", storage=st, tol=1e-300, max_cycles=10, cycles_per_launch=1)
        with M.Multigrid(shape, hfm._lib.OP_SIGMA7, cfg, slots=2) as h:
            for s in range(2):
                h.set_operator(hfm.ops.Sigma7(*(T.from_numpy(sig[k]).cuda() for k in range(3))),
                               slot=s)
                h.load(s, T.from_numpy(f).cuda())
            h.run(2)
            outs[st] = [h.fetch(s).cpu().numpy() for s in range(2)]
    for s in range(2):
        err = np.abs(outs[storage][s] - outs["f32"][s]).max() / np.abs(outs["f32"][s]).max()
        assert err < (3e-2 if storage == "bf16" else 5e-3), err
    np.testing.assert_array_equal(outs[storage][0], outs[storage][1])
