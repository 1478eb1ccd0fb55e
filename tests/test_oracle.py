"""CPU checks of the oracle: reference known-answers, TF layer semantics, golden fixtures."""
import json
import os

import numpy as np
import pytest

from oracle import mg, tfops, weights as W

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def pins():
    with open(os.path.join(GOLD, "reference_pins.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "oracle_small.npz"))


def test_reference_printed_kernel(pins):
    """Multigrid_3d_7point_source.ipynb cells 4, 5, 6, 10 at dt=0.1, D=(200,100,50)."""
    K = W.w2_7point(Dx=200.0, Dy=100.0, Dz=50.0, dt=0.1)
    assert K.sum() == pytest.approx(pins["sum_w2"], abs=1e-12)
    np.testing.assert_allclose(K[1], np.array(pins["centre_plane"]), atol=1e-12)
    assert K[1, 1, 1] == pytest.approx(pins["centre_weight"])
    np.testing.assert_allclose(K, np.array(pins["kernel_3x3x3"]), atol=1e-12)


def test_oracle_reproduces_reference_2d_cycle_values(pins):
    """The serial 2D run of ``notebooks/Parallel_multigrid_2D.ipynb`` (cell 20: 128^2,
    advection-diffusion weights of cell 5, 40x40 box as source and initial guess, restriction
    down to 2x2, one cycle) printed its 2x2 and 4x4 corrections (cells 50, 52).  The oracle's
    cycle gives the same numbers to the 8 printed decimals."""
    from oracle import kolmogorov as K2
    T = np.zeros((128, 128), np.float32)
    T[43:83, 43:83] = 1.0
    keep = {}
    K2.sawtooth2d(W.w2_2d_advection_diffusion(), T, T, 7, keep=keep)
    w = keep["w"]
    assert w[6].shape == (2, 2) and w[5].shape == (4, 4)
    np.testing.assert_allclose(w[6], np.array(pins["mg2d_w2"]), rtol=0, atol=6e-9)
    np.testing.assert_allclose(w[5], np.array(pins["mg2d_w4"]), rtol=0, atol=6e-9)


def _float32_dot_32_lanes(x):
    """sqrt(x . x) summed as a float32 BLAS dot with 4 x 8 fused multiply-add accumulators
    (element i lands in lane i mod 32; lanes added register by register, then across the 8
    lanes in order).  This is how the reference's ``np.linalg.norm`` of a float32 array is
    evaluated on an AVX2 host; the result differs from the exact norm in the 5th digit."""
    f = np.float32
    x = np.asarray(x, np.float64).ravel()
    acc = np.zeros(32, np.float32)
    for blk in x.reshape(-1, 32):
        acc = (acc.astype(np.float64) + blk * blk).astype(np.float32)
    a = acc.reshape(4, 8)
    v = (a[0] + a[1]) + (a[2] + a[3])
    h = f(0)
    for t in v:
        h = f(h + t)
    return f(np.sqrt(h))


def test_oracle_reproduces_reference_3d_solution_norm(pins):
    """The serial 3D run of ``notebooks/parallel_multigrid_advection_diffusion_3D.ipynb``
    (cell 15: 128^3, 7-point operator with Dx = Dy = Dz = 100, 40^3 box as source and initial
    guess, restriction down to 2^3 with two Jacobi sweeps there, 100 reference cycles)
    printed the norm of its float32 solution (cell 72): 288.47165.  The oracle's solution
    has that norm exactly when the norm is summed as the reference summed it, and within
    1e-4 exactly (the printed number's own rounding); the same cycle with one coarsest sweep
    misses by 3.6e-3, so the check separates the variants."""
    K = W.w2_7point(Dx=100.0, Dy=100.0, Dz=100.0, dt=1.0)
    assert K[1, 1, 1] == 600.0 and K[0, 1, 1] == -100.0
    ops = mg.hierarchy(mg.Stencil27(K), 7, 1.0)
    assert len(mg.level_shapes((128, 128, 128), min_edge=2)) == 7   # 128 ... 2
    T = np.zeros((128, 128, 128), np.float32)
    T[43:83, 43:83, 43:83] = 1.0
    want = pins["mg3d_norm_after_100"]

    def run(coarse_sweeps):
        v = T.copy()
        for _ in range(100):
            v = mg.sawtooth_cycle(ops, v, T, coarse_sweeps=coarse_sweeps)
        return v

    v = run(2)
    assert _float32_dot_32_lanes(v) == np.float32(want)
    exact = float(np.linalg.norm(v.astype(np.float64)))
    assert abs(exact - want) / want < 1e-4, exact
    one = float(np.linalg.norm(run(1).astype(np.float64)))
    assert abs(one - want) / want > 1e-3, one


def test_product_weights_match_oracle(pkg):
    w = pkg.weights
    np.testing.assert_allclose(w.anisotropic7(), W.w2_7point(), rtol=1e-7)
    np.testing.assert_allclose(w.anisotropic7(dt=0.1), W.w2_7point(dt=0.1), rtol=1e-6)
    np.testing.assert_allclose(w.pressure27(), W.w5_pressure27(), rtol=1e-6)
    np.testing.assert_allclose(w.diffusion27(0.1, 0.25), W.w1_diffusion27(0.1, 0.25), rtol=1e-6)
    for a, b in zip(w.advection(0.4, factor=0.5), W.advection_kernels(0.4, factor=0.5)):
        np.testing.assert_allclose(a, b, rtol=1e-6)
    for a, b in zip(w.divergence(0.1), W.divergence_kernels(0.1)):
        np.testing.assert_allclose(a, b, rtol=1e-6)
    assert w.pressure27()[1, 1, 1] == pytest.approx(88 / 26, rel=1e-6)
    np.testing.assert_allclose(w.advection_diffusion_2d(), W.w2_2d_advection_diffusion(), rtol=1e-12)
    # the 2D reference prints 'Sum up the weights of filter' = 1 (cell 3): the upwind and
    # diffusion terms cancel, the identity remains
    assert W.w2_2d_advection_diffusion().sum() == pytest.approx(1.0)


def test_param_counts(pins, pkg):
    """Keras summaries: 28 params for a 3x3x3 conv + bias, 9 for the 2x2x2 restriction."""
    ops = pytest.importorskip("torch") and pkg.ops
    assert ops.Conv3DSame(W.w2_7point()).count_params() == pins["params_conv3x3x3"]
    assert ops.Restriction().count_params() == pins["params_restrict2x2x2"]


@pytest.mark.parametrize("shape", [(1, 1, 1), (2, 3, 4), (5, 4, 7), (8, 8, 8)])
def test_conv_is_cross_correlation_with_zero_pad(shape):
    """Independent second opinion: torch CPU conv3d (cross-correlation, zero padding)."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape)
    K = rng.standard_normal((3, 3, 3))
    ref = torch.nn.functional.conv3d(torch.from_numpy(x)[None, None],
                                     torch.from_numpy(K)[None, None], padding=1)[0, 0].numpy()
    np.testing.assert_allclose(tfops.conv3d_same(x, K, np.float64), ref, rtol=1e-12, atol=1e-12)


def test_restrict_prolong_semantics():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(2)
    x = rng.standard_normal((7, 6, 9))
    ref = torch.nn.functional.avg_pool3d(torch.from_numpy(x)[None, None], 2)[0, 0].numpy()
    np.testing.assert_allclose(tfops.restrict_avg(x, np.float64), ref, rtol=1e-12)
    y = tfops.prolong_nearest(x[:3, :3, :3], np.float64)
    assert y.shape == (6, 6, 6)
    assert y[5, 4, 3] == x[2, 2, 1]
    # restriction is 1/8 of the prolongation's transpose
    a = rng.standard_normal((4, 4, 4))
    c = rng.standard_normal((2, 2, 2))
    lhs = (tfops.restrict_avg(a, np.float64) * c).sum()
    rhs = (a * tfops.prolong_nearest(c, np.float64)).sum() / 8.0
    assert lhs == pytest.approx(rhs, rel=1e-12)


def test_sigma_form_equals_directional_form():
    """Sigma7 (face means) equals the reference's six-array form with the same faces."""
    rng = np.random.default_rng(3)
    s = np.exp(rng.standard_normal((3, 5, 6, 7)))
    op = mg.Sigma7(s[0], s[1], s[2], dtype=np.float64)
    (xl, xh), (yl, yh), (zl, zh) = op.faces
    d = mg.Dir7({"xm": xl, "xp": xh, "ym": yl, "yp": yh, "zm": zl, "zp": zh}, op.diag, np.float64)
    x = rng.standard_normal((5, 6, 7))
    np.testing.assert_allclose(op.apply(x), d.apply(x), rtol=1e-12)
    # symmetric positive definite
    y = rng.standard_normal((5, 6, 7))
    assert (op.apply(x) * y).sum() == pytest.approx((x * op.apply(y)).sum(), rel=1e-10)
    assert (op.apply(x) * x).sum() > 0


def test_const7_is_sigma7_with_constant_sigma():
    rng = np.random.default_rng(4)
    x = rng.standard_normal((6, 5, 4))
    ones = np.ones((6, 5, 4))
    a = mg.Sigma7(200 * ones, 100 * ones, 50 * ones, dtype=np.float64).apply(x)
    b = mg.const7(50.0, 100.0, 200.0, dtype=np.float64).apply(x)
    # wall faces differ: SAME zero padding puts the ghost at distance h on both forms
    np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-9)


def test_golden_fixtures_reproduce(gold):
    """The oracle reproduces its committed fixtures bit-for-bit (regression pin)."""
    K7 = W.w2_7point()
    K27 = W.w5_pressure27()
    Kr = gold["kr"].astype(np.float64)
    for i in range(6):
        x, b, sig = gold["x_%d" % i], gold["b_%d" % i], gold["sig_%d" % i]
        np.testing.assert_array_equal(tfops.conv3d_same(x, K7), gold["conv_k7_%d" % i])
        np.testing.assert_array_equal(tfops.conv3d_same(x, K27), gold["conv_k27_%d" % i])
        np.testing.assert_allclose(tfops.conv3d_same(x, Kr), gold["conv_kr_%d" % i], rtol=1e-6, atol=1e-6)
        op = mg.Sigma7(sig[0], sig[1], sig[2])
        np.testing.assert_array_equal(op.apply(x), gold["sigma_apply_%d" % i])
        np.testing.assert_array_equal(mg.jacobi(op, x, b, 2.0 / 3.0), gold["sigma_jacobi_%d" % i])
        if "restrict_%d" % i in gold:
            np.testing.assert_array_equal(tfops.restrict_avg(x), gold["restrict_%d" % i])
        np.testing.assert_array_equal(tfops.prolong_nearest(x), gold["prolong_%d" % i])
    b = gold["saw7_b"]
    ops = mg.hierarchy(mg.Stencil27(K7), 5)
    phi = b.copy()
    for c in range(3):
        phi = mg.sawtooth_cycle(ops, phi, b)
        np.testing.assert_array_equal(phi, gold["saw7_after_%d" % (c + 1)])


def test_sawtooth_first_cycle_by_hand():
    """On 2^3 with two levels the reference cycle can be written out by hand."""
    K = W.w2_7point()
    d = K[1, 1, 1]
    b = np.arange(8, dtype=np.float64).reshape(2, 2, 2)
    ops = mg.hierarchy(mg.Stencil27(K, dtype=np.float64), 2)
    phi = b.copy()
    r = tfops.conv3d_same(phi, K, np.float64) - b
    w1 = r.mean() / d                     # restriction of the 2^3 block then J from zero on 1^3
    w = np.full((2, 2, 2), w1)
    w = w - tfops.conv3d_same(w, K, np.float64) / d + r / d
    p = phi - w
    p = p - tfops.conv3d_same(p, K, np.float64) / d + b / d
    np.testing.assert_allclose(mg.sawtooth_cycle(ops, phi, b), p, rtol=1e-12)


def test_vcycle_converges_and_pcg_faster(pkg):
    n = 16
    sig = pkg.problems.anisotropic_sigma((n, n, n), seed=0, log_std=1.0).astype(np.float64)
    f = pkg.problems.dipole((n, n, n), seed=0).astype(np.float64)
    op = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float64)
    ops = mg.hierarchy(op, len(mg.level_shapes((n, n, n))), 0.5)
    _, h = mg.solve(ops, f, mg.CycleConfig(), "V", 1e-6, 400)
    assert h[-1] < 1e-6
    assert all(b < a for a, b in zip(h, h[1:]))


def test_tomography_oracle_gradient_matches_finite_differences():
    """The float64 adjoint gradient of the oracle equals central differences of J."""
    from oracle import tomography as tomo
    rng = np.random.default_rng(5)
    n = 6
    logs = rng.normal(0, 0.5, (3, n, n, n))
    q = np.zeros((2, n, n, n))
    q[0, 2, 2, 2], q[0, 3, 4, 1] = 1, -1
    q[1, 4, 1, 3], q[1, 1, 3, 3] = 1, -1
    rec = np.array([1, 5, 9, 14, 20, 27, 33])
    d_obs = rng.normal(0, 0.01, (2, len(rec)))
    J, g, _ = tomo.misfit(np.exp(logs), q, rec, d_obs)
    eps = 1e-4  # the config's step; truncation error ~eps^2, roundoff ~1e-16 J / eps
    for (k, z, y, x) in [(0, 2, 2, 2), (1, 0, 3, 5), (2, 5, 0, 0), (0, 3, 4, 1), (2, 2, 2, 3)]:
        lp, lm = logs.copy(), logs.copy()
        lp[k, z, y, x] += eps
        lm[k, z, y, x] -= eps
        fd = (tomo.misfit(np.exp(lp), q, rec, d_obs, want_grad=False)[0]
              - tomo.misfit(np.exp(lm), q, rec, d_obs, want_grad=False)[0]) / (2 * eps)
        assert fd == pytest.approx(g[k, z, y, x], rel=1e-6, abs=1e-12 * abs(J))


def test_tomography_matrix_matches_operator():
    from oracle import tomography as tomo
    rng = np.random.default_rng(6)
    s = np.exp(rng.normal(0, 1, (3, 4, 5, 6)))
    x = rng.normal(0, 1, (4, 5, 6))
    A = tomo.assemble(s)
    ref = mg.Sigma7(s[0], s[1], s[2], dtype=np.float64).apply(x)
    np.testing.assert_allclose(A @ x.ravel(), ref.ravel(), rtol=1e-12, atol=1e-12)


# ------------------------------------------------------------------------------ 2D path
def test_conv2d_matches_torch_zero_and_periodic():
    import torch
    from oracle import kolmogorov as K2
    rng = np.random.default_rng(21)
    x = rng.standard_normal((9, 14)).astype(np.float32)
    w = rng.standard_normal((3, 3)).astype(np.float32)
    t = torch.from_numpy(x)[None, None]
    k = torch.from_numpy(w)[None, None]
    zero = torch.nn.functional.conv2d(t, k, padding=1)[0, 0].numpy()
    wrap = torch.nn.functional.conv2d(torch.nn.functional.pad(t, (1, 1, 1, 1), mode="circular"), k)[0, 0].numpy()
    np.testing.assert_allclose(K2.conv2d(x, w), zero, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(K2.conv2d(x, w, periodic=True), wrap, rtol=1e-5, atol=1e-5)


def test_2d_reference_cycle_converges():
    """Multigrid_2D.ipynb#c18 on its own problem (128^2, box source of 40 x 40 ones at
    (43, 43)): the residual falls cycle after cycle."""
    from oracle import kolmogorov as K2
    w = W.w2_2d_advection_diffusion()
    b = np.zeros((128, 128), np.float32)
    b[43:83, 43:83] = 1.0
    v = b.copy()
    res = []
    for _ in range(5):
        v = K2.sawtooth2d(w, v, b, len(K2.level_shapes((128, 128), 1)))
        res.append(np.linalg.norm(K2.conv2d(v, w) - b))
    assert all(r1 < r0 for r0, r1 in zip(res, res[1:]))


def test_periodic_vcycle_contracts():
    from oracle import kolmogorov as K2
    n = 64
    rng = np.random.default_rng(3)
    f = rng.standard_normal((n, n))
    f -= f.mean()
    mg = K2.VCycle2D(K2.laplace5(2 * np.pi / n), (n, n))
    p = np.zeros((n, n))
    r0 = mg.rel_residual(p, f)
    p = mg.solve(p, f, 4)
    assert mg.rel_residual(p, f) < 1e-3 * r0
    assert abs(p.mean()) < 1e-12


def test_mesh_mask_follows_reference_loop(pkg):
    """ns.mask_from_mesh against the reference's loop (naiver_stokes_3D.py:560-564) on a
    synthetic mesh array."""
    pytest.importorskip("torch")
    ns = pkg.ns
    nx, ny, nz = 12, 10, 8
    rng = np.random.default_rng(4)
    mesh = (rng.random((1, nx + 32, ny + 32, nz, 1)) > 0.3).astype(np.float64)
    ref = np.zeros((1, nz, ny, nx, 1))
    for i in range(1, nx - 1):
        for j in range(1, ny - 1):
            for k in range(1, nz - 1):
                if mesh[0][i + 16][j + 16][k][0] == 0:
                    ref[0][k][j][i][0] = 100000
    got = ns.mask_from_mesh(mesh, (nz, ny, nx), device="cpu").numpy()
    np.testing.assert_array_equal(got, ref[0, ..., 0])


def test_load_mesh_mask_reads_reference_mesh_file(pkg, tmp_path):
    """ns.load_mesh_mask on a mesh_<n>_sk.npy-style file written here: the file's array goes
    through the reference's loop (naiver_stokes_3D.py:527, 560-564) unchanged."""
    pytest.importorskip("torch")
    ns = pkg.ns
    nx, ny, nz = 10, 9, 6
    rng = np.random.default_rng(11)
    mesh = (rng.random((1, nx + 32, ny + 32, nz + 3, 1)) > 0.4).astype(np.float32)
    path = tmp_path / "mesh_10_sk.npy"
    np.save(path, mesh)
    ref = np.zeros((nz, ny, nx))
    for i in range(1, nx - 1):
        for j in range(1, ny - 1):
            for k in range(1, nz - 1):
                if mesh[0][i + 16][j + 16][k][0] == 0:
                    ref[k][j][i] = 100000
    got = ns.load_mesh_mask(str(path), (nz, ny, nx), device="cpu").numpy()
    assert got.dtype == np.float32
    np.testing.assert_array_equal(got, ref)
    assert (got > 0).sum() > 0
