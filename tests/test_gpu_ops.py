"""GPU parity of the stateless operators (C ABI via ctypes) against the oracle.

Tolerance: float32 kernels vs the float32 oracle within 1e-5 relative to the field's max
(the reference-parity bar); the ordering of float32 sums differs, nothing else.
"""
import os

import numpy as np
import pytest

from oracle import mg, tfops, weights as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
RTOL = 1e-5

# X % 4 == 0 grids run the plane-marching kernels, the others the generic ones; X = 132
# (33 vectors per row) makes rows straddle warp boundaries, Z = 70 spans several z-chunks.
SHAPES = [(1, 1, 1), (2, 2, 2), (3, 5, 4), (4, 4, 4), (5, 7, 6), (8, 6, 10), (16, 16, 16),
          (12, 20, 32), (32, 8, 64), (9, 33, 40), (70, 18, 132), (64, 40, 96)]


def close(got, ref, rtol=RTOL, operands=()):
    """max |got - ref| <= rtol * scale, scale = the largest magnitude among the result and
    the operands (float32 rounding of x - A x / d is bounded by the operands' size, which
    can exceed the result's on 1^3 and 2^3 grids)."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    scale = max([np.abs(ref).max(), 1e-30] + [float(np.abs(np.asarray(o)).max()) for o in operands])
    err = np.abs(got - ref).max() / scale
    assert err <= rtol, "max rel err %.3e > %.1e" % (err, rtol)


@pytest.fixture(scope="module")
def T(hfm):
    import torch
    return torch


def dev(T, a):
    return T.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


@pytest.mark.parametrize("shape", SHAPES)
def test_conv3d_matches_oracle(hfm, T, shape):
    rng = np.random.default_rng(hash(shape) % 2 ** 32)
    x = rng.standard_normal(shape).astype(np.float32)
    for K in (W.w2_7point(), W.w5_pressure27(), rng.standard_normal((3, 3, 3))):
        y = hfm.ops.conv3d_same(dev(T, x), K).cpu().numpy()
        close(y, tfops.conv3d_same(x, K, np.float64))


def test_golden_fixtures(hfm, T):
    g = np.load(os.path.join(GOLD, "oracle_small.npz"))
    ops = hfm.ops
    for i in range(6):
        x, b, sig = g["x_%d" % i], g["b_%d" % i], g["sig_%d" % i]
        close(ops.conv3d_same(dev(T, x), W.w2_7point()).cpu(), g["conv_k7_%d" % i])
        close(ops.conv3d_same(dev(T, x), W.w5_pressure27()).cpu(), g["conv_k27_%d" % i])
        close(ops.conv3d_same(dev(T, x), g["kr"]).cpu(), g["conv_kr_%d" % i])
        sx, sy, sz = (dev(T, sig[k]) for k in range(3))
        op = ops.Sigma7(sx, sy, sz)
        close(ops.apply(op, dev(T, x)).cpu(), g["sigma_apply_%d" % i])
        close(ops.jacobi(op, dev(T, x), dev(T, b), 2.0 / 3.0).cpu(), g["sigma_jacobi_%d" % i],
              operands=(x, b))
        close(ops.jacobi(ops.Stencil27(W.w2_7point()), dev(T, x), dev(T, b), 1.0).cpu(),
              g["k7_jacobi_ref_%d" % i], operands=(x, b))
        if "restrict_%d" % i in g:
            np.testing.assert_allclose(ops.restrict_avg(dev(T, x)).cpu().numpy(),
                                       g["restrict_%d" % i], rtol=1e-6, atol=1e-7)
        np.testing.assert_array_equal(ops.prolong_nearest(dev(T, x)).cpu().numpy(),
                                      g["prolong_%d" % i])


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("form", ["const7", "sigma7", "dir7", "k27"])
def test_apply_residual_jacobi(hfm, T, shape, form):
    rng = np.random.default_rng(7)
    x = rng.standard_normal(shape).astype(np.float32)
    b = rng.standard_normal(shape).astype(np.float32)
    ops = hfm.ops
    if form == "const7":
        gop, oop = ops.Const7(50.0, 100.0, 200.0), mg.const7(50.0, 100.0, 200.0, dtype=np.float64)
    elif form == "k27":
        gop, oop = ops.Stencil27(W.w5_pressure27()), mg.Stencil27(W.w5_pressure27(), dtype=np.float64)
    else:
        sig = np.exp(rng.standard_normal((3,) + shape)).astype(np.float32)
        if form == "sigma7":
            gop = ops.Sigma7(*(dev(T, sig[k]) for k in range(3)))
            oop = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float64)
        else:
            s7 = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float32)
            (xl, xh), (yl, yh), (zl, zh) = s7.faces
            arrs = {"xm": xl, "xp": xh, "ym": yl, "yp": yh, "zm": zl, "zp": zh, "tot": s7.diag}
            gop = ops.Dir7({k: dev(T, v) for k, v in arrs.items()})
            oop = mg.Dir7({k: v for k, v in arrs.items() if k != "tot"}, arrs["tot"], np.float64)
    xd, bd = dev(T, x), dev(T, b)
    close(ops.apply(gop, xd).cpu(), oop.apply(x))
    close(ops.residual(gop, xd, bd).cpu(), mg.residual(oop, x, b))
    close(ops.jacobi(gop, xd, bd, 0.8).cpu(), mg.jacobi(oop, x, b, 0.8))
    ref = x.astype(np.float64)
    for _ in range(3):
        ref = mg.jacobi(oop, ref, b, 2.0 / 3.0)
    close(ops.jacobi(gop, xd, bd, 2.0 / 3.0, sweeps=3).cpu(), ref)
    close(ops.jacobi(gop, None, bd, 2.0 / 3.0).cpu(), mg.jacobi(oop, np.zeros_like(x), b, 2.0 / 3.0))


def test_flags(hfm, T):
    ops, L = hfm.ops, hfm._lib
    rng = np.random.default_rng(9)
    s = (6, 5, 8)
    x = rng.standard_normal(s).astype(np.float32)
    b = rng.standard_normal(s).astype(np.float32)
    K = W.w5_pressure27()
    gop, oop = ops.Stencil27(K), mg.Stencil27(K, dtype=np.float64)
    r = ops.residual(gop, dev(T, x), dev(T, b), flags=L.FLAG_ZERO_XEND).cpu().numpy()
    ref = mg.residual(oop, x, b)
    ref[..., -1] = 0
    close(r, ref)
    xz = x.copy()
    xz[..., -1] = 0
    close(ops.jacobi(gop, dev(T, x), dev(T, b), 1.0, flags=L.FLAG_ZERO_XEND).cpu(),
          mg.jacobi(oop, xz, b, 1.0))
    j = mg.jacobi(oop, x, b, 1.0)
    j[0] = j[1]
    close(ops.jacobi(gop, dev(T, x), dev(T, b), 1.0, flags=L.FLAG_TOP_COPY).cpu(), j)


@pytest.mark.parametrize("shape", [(2, 2, 2), (4, 6, 8), (16, 16, 16), (32, 8, 64), (10, 12, 14),
                                   (70, 18, 132), (64, 40, 96)])
def test_fused_transfer_kernels(hfm, T, shape):
    ops = hfm.ops
    rng = np.random.default_rng(11)
    x = rng.standard_normal(shape).astype(np.float32)
    b = rng.standard_normal(shape).astype(np.float32)
    sig = np.exp(rng.standard_normal((3,) + shape)).astype(np.float32)
    gop = ops.Sigma7(*(dev(T, sig[k]) for k in range(3)))
    oop = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float64)
    rc, rf = ops.residual_restrict(gop, dev(T, x), dev(T, b), want_fine=True)
    r = mg.residual(oop, x, b)
    close(rf.cpu(), r)
    close(rc[0].cpu(), tfops.restrict_avg(r, np.float64))
    c = rng.standard_normal(tuple(v // 2 for v in shape)).astype(np.float32)
    out = ops.prolong_correct_smooth(gop, dev(T, x), dev(T, c), dev(T, b), 2.0 / 3.0)
    close(out.cpu(), mg.jacobi(oop, x - tfops.prolong_nearest(c, np.float64), b, 2.0 / 3.0))
    out = ops.prolong_correct_smooth(gop, None, dev(T, c), dev(T, b), 1.0)
    close(out.cpu(), mg.jacobi(oop, tfops.prolong_nearest(c, np.float64), b, 1.0))


@pytest.mark.parametrize("s", [(8, 12, 16), (10, 12, 14)])
def test_batched_equals_single(hfm, T, s):
    ops = hfm.ops
    rng = np.random.default_rng(12)
    B = 5
    x = rng.standard_normal((B,) + s).astype(np.float32)
    sig = np.exp(rng.standard_normal((3, B) + s)).astype(np.float32)
    gop = ops.Sigma7(*(dev(T, sig[k]) for k in range(3)))
    yb = ops.apply(gop, dev(T, x)).cpu().numpy()
    for i in range(B):
        gi = ops.Sigma7(*(dev(T, sig[k, i]) for k in range(3)))
        np.testing.assert_array_equal(yb[i], ops.apply(gi, dev(T, x[i])).cpu().numpy())


def test_reductions(hfm, T):
    ops = hfm.ops
    rng = np.random.default_rng(13)
    x = rng.standard_normal((3, 70000)).astype(np.float32)
    n = ops.norm2(dev(T, x)).cpu().numpy()
    np.testing.assert_allclose(n, np.linalg.norm(x.astype(np.float64), axis=1), rtol=1e-12)
    m = ops.max_abs(dev(T, x)).cpu().numpy()
    np.testing.assert_array_equal(m, np.abs(x).max(axis=1))
    # deterministic: same bits on repeat
    assert ops.norm2(dev(T, x)).cpu().numpy().tobytes() == n.tobytes()


def test_bad_shapes_raise(hfm, T):
    ops = hfm.ops
    with pytest.raises(ValueError):
        ops.conv3d_same(T.zeros((2, 2), device="cuda"), W.w2_7point())
    with pytest.raises(hfm._lib.HfmError):
        ops.restrict_avg(T.zeros((1, 1, 1), device="cuda"))


@pytest.mark.parametrize("storage", ["bf16", "f16"])
def test_reduced_precision_storage_smoother(hfm, T, storage):
    """The handle's bf16 / fp16 storage path: one V-cycle agrees with the float32 handle to
    the storage precision."""
    n = 32
    sig = hfm.problems.anisotropic_sigma((n, n, n), seed=2, log_std=1.0)
    f = hfm.problems.dipole((n, n, n), seed=2)
    M = hfm.multigrid
    outs = {}
    for st in ("f32", storage):
        cfg = M.SolverConfig(cycle="V", storage=st, tol=1e-300, max_cycles=10, cycles_per_launch=1)
        with M.Multigrid((n, n, n), hfm._lib.OP_SIGMA7, cfg, slots=1) as h:
            h.set_operator(ops_sigma(hfm, T, sig))
            h.load(0, dev(T, f))
            h.run(2)
            outs[st] = h.fetch(0).cpu().numpy()
    err = np.abs(outs[storage] - outs["f32"]).max() / np.abs(outs["f32"]).max()
    assert err < (3e-2 if storage == "bf16" else 5e-3), err


def ops_sigma(hfm, T, sig):
    return hfm.ops.Sigma7(*(dev(T, sig[k]) for k in range(3)))


@pytest.mark.parametrize("shape", [(3, 17, 24, 64), (2, 16, 9, 40), (1, 6, 6, 14)])
def test_transfers_vector_and_scalar_paths(hfm, T, shape):
    """Restriction and prolongation on batched grids whose rows take the 16-byte vector
    kernels (X a multiple of 4) and one that does not (X = 14), odd Z / Y floored: against
    the oracle's VALID average (same summation order: the bits of the float32 oracle) and
    UpSampling3D (exact)."""
    ops = hfm.ops
    rng = np.random.default_rng(23)
    x = rng.standard_normal(shape).astype(np.float32)
    got = ops.restrict_avg(dev(T, x)).cpu().numpy()
    np.testing.assert_array_equal(got, tfops.restrict_avg(x, np.float32))
    up = ops.prolong_nearest(dev(T, x)).cpu().numpy()
    np.testing.assert_array_equal(up, tfops.prolong_nearest(x))
