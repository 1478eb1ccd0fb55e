"""The persistent small-end kernel: the V-cycle level above the fused coarse cycle (when the
plane-marching TMA kernels do not take it) and the coarse cycle itself, for every slot of a
handle, in one launch that walks an (instance, step, tile) work list.

Checked against the separate launches (without HFM_OPT_PERSISTENT) and the oracle: stationary
V-cycles to the float32 evaluation error, solves to tolerance with the same iteration
counts, and the bounded dependency waits: with a wait budget of zero every wait expires, the
slots end with HFM_ERR_TIMEOUT, and the next handle solves normally.
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


def _problems(hfm, n, B, seed, log_std=1.0):
    sig = np.stack([hfm.problems.anisotropic_sigma((n, n, n), seed=seed + i, log_std=log_std)
                    for i in range(B)], axis=1)
    f = np.stack([hfm.problems.dipole((n, n, n), seed=seed + i) for i in range(B)])
    return sig, f


@pytest.mark.parametrize("n", [64, 96])
def test_vcycles_match_separate_launches_and_oracle(hfm, T, n):
    """Stationary V(2,2) cycles on 8 slots (fine level on the TMA kernels, the level below on
    the persistent kernel): against the separate launches and the float32 oracle cycle."""
    M, L = hfm.multigrid, hfm._lib
    B = 8
    sig, f = _problems(hfm, n, B, 40)
    outs = {}
    for persistent in (True, False):
        cfg = M.SolverConfig(cycle="V", tol=1e-300, max_cycles=10, cycles_per_launch=1,
                             persistent=persistent)
        with M.Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=B) as h:
            h.set_operator(hfm.ops.Sigma7(*(T.from_numpy(np.ascontiguousarray(sig[k])).cuda() for k in range(3))))
            for s in range(B):
                h.load(s, T.from_numpy(f[s]).cuda())
            h.run(1)
            outs[persistent] = [h.fetch(s).cpu().numpy() for s in range(B)]
    shapes = mg.level_shapes((n, n, n))
    ccfg = mg.CycleConfig(2, 2, 2.0 / 3.0, 32)
    for s in (0, B - 1):
        ops = mg.hierarchy(mg.Sigma7(sig[0, s], sig[1, s], sig[2, s], dtype=np.float64), len(shapes), 0.5)
        ref = mg.vcycle(ops, 0, np.zeros((n, n, n)), f[s].astype(np.float64), ccfg)
        scale = np.abs(ref).max()
        assert np.abs(outs[True][s] - ref).max() <= 2e-5 * scale
        assert np.abs(outs[True][s] - outs[False][s]).max() <= 2e-5 * scale


@pytest.mark.parametrize("storage,n", [("f32", 32), ("bf16", 32), ("bf16", 48), ("f16", 64)])
def test_solves_match_separate_launches(hfm, T, storage, n):
    """PCG (float32) or float64 refinement (16-bit) with the persistent small end on 8 slots -
    at 32^3 the whole preconditioner V-cycle is one persistent launch, its last sweep summing
    r . z - reaches 1e-6 in the separate launches' iteration counts: within 2 in float32;
    with 16-bit inner cycles within 20 %, since the persistent kernel keeps the first
    sweep's iterate in float32 where the separate launches store it in the storage type,
    and the inner CG's counts move with such roundings."""
    M, L = hfm.multigrid, hfm._lib
    B = 8
    sig, f = _problems(hfm, n, B, 50, log_std=1.5)
    accel = "cg" if storage == "f32" else "ir"
    res = {}
    for persistent in (True, False):
        cfg = M.SolverConfig(cycle="V", accel=accel, storage=storage, tol=1e-6, max_cycles=600,
                             inner_tol=1e-3, persistent=persistent)
        with M.Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=B) as h:
            h.set_operator(hfm.ops.Sigma7(*(T.from_numpy(np.ascontiguousarray(sig[k])).cuda() for k in range(3))))
            for s in range(B):
                h.load(s, T.from_numpy(f[s]).cuda())
            for _ in range(400):
                h.run(4)
                st = h.query()
                if not any(x["active"] for x in st):
                    break
            xs = [(h.fetch_f64(s) if accel == "ir" else h.fetch(s)).double().cpu().numpy() for s in range(B)]
            res[persistent] = (xs, st)
    for s in range(B):
        x, st = res[True][0][s], res[True][1][s]
        assert st["status"] == 0, (s, st)
        op64 = mg.Sigma7(sig[0, s], sig[1, s], sig[2, s], dtype=np.float64)
        assert mg.rel_residual(op64, x, f[s]) < 1.5e-6
        c1, c0 = st["cycles"], res[False][1][s]["cycles"]
        band = 2 if storage == "f32" else max(2, 0.2 * c0)
        assert abs(c1 - c0) <= band, (s, st, res[False][1][s])


def test_expired_dependency_waits_end_slots_with_timeout(hfm, T):
    """32^3 on 8 slots has no TMA level: the only bounded waits are the persistent kernel's
    dependency waits.  With a wait budget of zero they expire, the slots end with
    HFM_ERR_TIMEOUT, no kernel hangs, and a new handle with the normal budget solves."""
    M, L = hfm.multigrid, hfm._lib
    n, B = 32, 8
    sig, f = _problems(hfm, n, B, 60)
    op = hfm.ops.Sigma7(*(T.from_numpy(np.ascontiguousarray(sig[k])).cuda() for k in range(3)))
    fd = T.from_numpy(f).cuda()
    cfg = M.SolverConfig(cycle="V", accel="cg", tol=1e-6, max_cycles=40, persistent=True)
    cnt, drain = C.c_int(0), C.c_int(0)
    L.call("hfm_device_timeouts", C.byref(cnt), 1)
    L.call("hfm_device_drain_timeouts", C.byref(drain), 1)
    L.call("hfm_set_wait_budget", 0)
    try:
        with M.Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=B) as h:
            h.set_operator(op)
            _, stats = h.solve(fd)
    finally:
        L.call("hfm_set_wait_budget", 1 << 20)
    L.call("hfm_device_timeouts", C.byref(cnt), 1)
    L.call("hfm_device_drain_timeouts", C.byref(drain), 1)
    assert cnt.value > 0
    assert [s["status"] for s in stats] == [L.ERR_TIMEOUT] * B, stats
    with M.Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=B) as h:
        h.set_operator(op)
        phi, stats = h.solve(fd)
    assert [s["status"] for s in stats] == [L.OK] * B, stats
    L.call("hfm_device_timeouts", C.byref(cnt), 0)
    assert cnt.value == 0
