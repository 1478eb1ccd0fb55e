"""Reference runs replayed on the GPU, against what the reference printed.

``notebooks/Parallel_multigrid_2D.ipynb`` cell 20 runs one serial 2D sawtooth cycle on 128^2
(the cell-5 advection-diffusion weights, a 40 x 40 box of ones at offset 43 as both source
and initial guess, restriction down to 2 x 2); cells 50 and 52 printed the 2 x 2 and 4 x 4
corrections to 8 decimals.  ``kolmogorov.Multigrid2D.sawtooth`` runs that cycle; its
corrections are checked to 1e-8 (the last printed digit; a few float32 ulps of values near
0.02).

``notebooks/parallel_multigrid_advection_diffusion_3D.ipynb`` cell 15 runs 100 serial
sawtooth cycles on 128^3: the 7-point operator with Dx = Dy = Dz = 100 (centre 600), a 40^3
box of ones at offset 43 as both source and initial guess, restriction down to 2^3 with two
Jacobi sweeps there, one on each finer level, the fine correction and one Jacobi on the
iterate.  Cell 72 printed the norm of the float32 solution: 288.47165.  The loop below is the
notebook's, with its ``CNN3D_A_<n>`` / ``CNN3D_res_<n>`` / ``CNN3D_prol_<n>`` models replaced
by ``ops.Conv3DSame`` / ``ops.Restriction`` / ``ops.Prolongation`` (one object serves every
size) and its arithmetic written in the same order.  The printed norm carries the rounding of
a float32 ``np.linalg.norm`` (5e-5 here), so the exact norm is checked to 1e-4; the solution
is also checked against the pinned oracle's to 1e-5 of its largest value.  The same run goes
through the multigrid handle too (``SolverConfig.reference(coarse_sweeps=2)``).
"""
import json
import os

import numpy as np
import pytest

from oracle import kolmogorov as K2, mg as M, weights as OW

pytestmark = pytest.mark.gpu


def _printed():
    with open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")) as fh:
        return json.load(fh)


def test_2d_cycle_printed_corrections(hfm):
    import torch
    pins = _printed()
    mg = hfm.kolmogorov.Multigrid2D((128, 128), hfm.weights.advection_diffusion_2d(),
                                    storage="f32", periodic=False, coarse_scale=1.0, min_edge=2,
                                    omega=1.0)
    assert mg.L == 7 and mg.shapes[-1] == (2, 2)
    b = np.zeros((128, 128), np.float32)
    b[43:83, 43:83] = 1.0
    bd = torch.from_numpy(b).cuda().view(1, 128, 128)
    v = mg.sawtooth(bd.clone(), bd)
    np.testing.assert_allclose(mg.w[6][0].cpu().numpy(), np.array(pins["mg2d_w2"]), rtol=0,
                               atol=1e-8)
    np.testing.assert_allclose(mg.w[5][0].cpu().numpy(), np.array(pins["mg2d_w4"]), rtol=0,
                               atol=1e-8)
    ref = K2.sawtooth2d(OW.w2_2d_advection_diffusion(), b, b, 7)
    err = np.abs(v[0].cpu().numpy() - ref).max() / np.abs(ref).max()
    assert err < 1e-5, err


_ORACLE_3D = {}


def _oracle_3d(w2):
    """The pinned oracle's solution of the 3D serial run (computed once per session)."""
    if "v" not in _ORACLE_3D:
        n = 128
        Tn = np.zeros((n, n, n), np.float32)
        Tn[43:83, 43:83, 43:83] = 1.0
        hier = M.hierarchy(M.Stencil27(w2), 7, 1.0)
        v = Tn.copy()
        for _ in range(100):
            v = M.sawtooth_cycle(hier, v, Tn, coarse_sweeps=2)
        _ORACLE_3D["v"] = v
    return _ORACLE_3D["v"]


def test_advection_diffusion_3d_serial_run(hfm):
    import torch
    ops, W = hfm.ops, hfm.weights
    printed = _printed()["mg3d_norm_after_100"]
    w2 = W.anisotropic7(Dx=100.0, Dy=100.0, Dz=100.0)
    d = float(w2[1, 1, 1])
    assert d == 600.0
    A, res, prol = ops.Conv3DSame(w2), ops.Restriction(), ops.Prolongation()
    n = 128
    T = torch.zeros((1, n, n, n, 1), device="cuda")
    T[0, 43:83, 43:83, 43:83, 0] = 1.0
    values, b = T.clone(), T
    for _ in range(100):
        w = torch.zeros((1, 2, 2, 2, 1), device="cuda")
        r = A(values) - b
        rs = [r]
        for _ in range(6):                       # r_64 ... r_2
            rs.append(res(rs[-1]))
        for _ in range(2):                       # two sweeps on 2^3
            w = w - A(w) / d + rs[6] / d
        for lvl in range(5, 0, -1):              # 4^3 ... 64^3
            w = prol(w)
            w = w - A(w) / d + rs[lvl] / d
        w = prol(w)
        w = w - A(w) / d + r / d
        values = values - w
        values = values - A(values) / d + b / d
    got = values[0, :, :, :, 0].double()
    norm = float(got.norm())
    assert abs(norm - printed) / printed < 1e-4, norm

    v = _oracle_3d(w2)
    err = np.abs(got.cpu().numpy() - v).max() / np.abs(v).max()
    assert err < 1e-5, err


def test_advection_diffusion_3d_serial_run_on_the_handle(hfm):
    """The same run through the multigrid handle (``hfm_mg_*``: the sawtooth cycle with two
    coarsest sweeps, 100 cycles captured in CUDA graphs)."""
    import torch
    Mg, W = hfm.multigrid, hfm.weights
    printed = _printed()["mg3d_norm_after_100"]
    w2 = W.anisotropic7(Dx=100.0, Dy=100.0, Dz=100.0)
    n = 128
    T = torch.zeros((1, n, n, n), device="cuda")
    T[0, 43:83, 43:83, 43:83] = 1.0
    # max_cycles above the 100 run, so that the slot stays active through the last one
    cfg = Mg.SolverConfig.reference(n_levels=7, cycles=102, coarse_sweeps=2)
    with Mg.Multigrid((n, n, n), hfm._lib.OP_K27, cfg, slots=1) as h:
        assert h.levels[-1] == (2, 2, 2)
        h.set_operator(hfm.ops.Stencil27(w2))
        h.load(0, T, T)
        h.run(100)
        got = h.fetch(0).double()
    norm = float(got.norm())
    assert abs(norm - printed) / printed < 1e-4, norm
    v = _oracle_3d(w2)
    err = np.abs(got.cpu().numpy() - v).max() / np.abs(v).max()
    assert err < 1e-5, err
