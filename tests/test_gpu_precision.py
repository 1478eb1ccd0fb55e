"""Mixed-precision iterative refinement (accel="ir") on the GPU.

The inner V-cycles store fields and conductivities in float32 / bf16 / fp16 (float32
arithmetic); the outer residual, its norm and the solution update run in float64.  Each
solve must reach a *true* relative residual (recomputed here in float64 by the oracle)
below the tolerance; the error against the float64 oracle solution is bounded too.
"""
import numpy as np
import pytest

from oracle import mg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T(hfm):
    import torch
    return torch


def _solve(hfm, T, n, seed, log_std, storage, tol=1e-6, f64_io=False):
    M = hfm.multigrid
    sig = hfm.problems.anisotropic_sigma((n, n, n), seed=seed, log_std=log_std)
    f = hfm.problems.dipole((n, n, n), seed=seed)
    cfg = M.SolverConfig(cycle="V", accel="ir", storage=storage, tol=tol, max_cycles=600)
    with M.Multigrid((n, n, n), hfm._lib.OP_SIGMA7, cfg, slots=1) as h:
        h.set_operator(hfm.ops.Sigma7(*(T.from_numpy(sig[k]).cuda() for k in range(3))))
        if f64_io:
            h.load_f64(0, T.from_numpy(f.astype(np.float64)).cuda())
        else:
            h.load(0, T.from_numpy(f).cuda())
        for _ in range(200):
            h.run(4)
            st = h.query()[0]
            if not st["active"]:
                break
        x = h.fetch_f64(0).cpu().numpy()
    return sig, f, x, st


@pytest.mark.parametrize("storage", ["f32", "bf16", "f16"])
@pytest.mark.parametrize("log_std", [1.0, 2.0])
def test_refinement_reaches_true_tolerance(hfm, T, storage, log_std):
    n = 32
    sig, f, x, st = _solve(hfm, T, n, 3, log_std, storage)
    assert st["status"] == 0, st
    op64 = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float64)
    rel = mg.rel_residual(op64, x, f)
    assert rel < 1e-6, (storage, log_std, rel, st)
    # the reported residual is the float64 outer residual
    assert abs(rel - st["rel_resid"]) <= 1e-9 + 1e-3 * rel
    ops64 = mg.hierarchy(op64, len(mg.level_shapes((n, n, n))), 0.5)
    x64, _ = mg.pcg_solve(ops64, f.astype(np.float64), mg.CycleConfig(), tol=1e-12)
    err = np.linalg.norm(x - x64) / np.linalg.norm(x64)
    # the error is bounded by the condition number times the residual
    assert err < 1e-3, err


def test_refinement_tighter_than_float32(hfm, T):
    """1e-10 relative residual (beyond float32 arithmetic) with float64 right-hand side."""
    n = 32
    sig, f, x, st = _solve(hfm, T, n, 4, 1.0, "bf16", tol=1e-10, f64_io=True)
    assert st["status"] == 0, st
    op64 = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float64)
    assert mg.rel_residual(op64, x, f) < 1e-10
    assert st["outer"] >= 2
