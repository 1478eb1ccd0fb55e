"""Failure path of the bounded device waits, without faulting or hanging the GPU: with a wait
budget of zero every TMA plane wait expires at once; the kernels stop, let the copies they
issued land, count the timeout and return.  The host reads the count, the context stays
usable, and the next call with the normal budget is correct."""
import ctypes as C

import numpy as np
import pytest

from oracle import mg

pytestmark = pytest.mark.gpu


def test_expired_waits_are_counted_and_the_context_survives(hfm):
    import torch
    L, ops = hfm._lib, hfm.ops
    rng = np.random.default_rng(17)
    shape = (2, 16, 32, 64)  # TMA-eligible: X >= 48, Y >= 8
    x = rng.standard_normal(shape).astype(np.float32)
    b = rng.standard_normal(shape).astype(np.float32)
    sig = np.exp(rng.standard_normal((3,) + shape)).astype(np.float32)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    op = ops.Sigma7(d(sig[0]), d(sig[1]), d(sig[2]))
    cnt = C.c_int(0)
    L.call("hfm_device_timeouts", C.byref(cnt), 1)  # clear
    L.call("hfm_set_wait_budget", 0)
    try:
        ops.jacobi(op, d(x), d(b), 0.8)
        torch.cuda.synchronize()
    finally:
        L.call("hfm_set_wait_budget", 1 << 20)
    L.call("hfm_device_timeouts", C.byref(cnt), 1)
    assert cnt.value > 0
    with pytest.raises(L.HfmError):
        L.call("hfm_set_wait_budget", -1)
    # the same call with the normal budget: no timeout, the oracle's answer
    y = ops.jacobi(op, d(x), d(b), 0.8).cpu().numpy()
    L.call("hfm_device_timeouts", C.byref(cnt), 0)
    assert cnt.value == 0
    for i in range(shape[0]):
        oop = mg.Sigma7(sig[0, i], sig[1, i], sig[2, i], dtype=np.float64)
        ref = mg.jacobi(oop, x[i].astype(np.float64), b[i].astype(np.float64), 0.8)
        assert np.abs(y[i] - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("accel,storage", [("cg", "f32"), ("ir", "bf16")])
def test_handle_reports_timeout_after_expired_waits(hfm, accel, storage):
    """A solve whose TMA waits expire ends every slot with HFM_ERR_TIMEOUT (never with a status
    computed from an incomplete stage); after the counters are cleared a new handle solves."""
    import torch
    L, M, ops = hfm._lib, hfm.multigrid, hfm.ops
    n, B = 64, 2  # TMA-eligible fine level
    sig = np.stack([hfm.problems.anisotropic_sigma((n, n, n), seed=5 + i, log_std=1.0)
                    for i in range(B)], axis=1)
    f = np.stack([hfm.problems.dipole((n, n, n), seed=5 + i) for i in range(B)])
    sd = torch.from_numpy(sig).cuda()
    fd = torch.from_numpy(f).cuda()
    op = ops.Sigma7(sd[0], sd[1], sd[2])
    cfg = M.SolverConfig(cycle="V", accel=accel, storage=storage, tol=1e-6, max_cycles=60)
    cnt, drain = C.c_int(0), C.c_int(0)
    L.call("hfm_device_timeouts", C.byref(cnt), 1)
    L.call("hfm_device_drain_timeouts", C.byref(drain), 1)
    L.call("hfm_set_wait_budget", 0)  # graphs captured from here on carry budget 0
    try:
        with M.Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=B) as h:
            h.set_operator(op)
            _, stats = h.solve(fd)
    finally:
        L.call("hfm_set_wait_budget", 1 << 20)
    L.call("hfm_device_timeouts", C.byref(cnt), 1)
    L.call("hfm_device_drain_timeouts", C.byref(drain), 1)
    assert cnt.value > 0 and drain.value == 0
    assert [s["status"] for s in stats] == [L.ERR_TIMEOUT] * B, stats
    assert not any(s["active"] for s in stats)
    with M.Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=B) as h:
        h.set_operator(op)
        phi, stats = h.solve(fd)
    assert [s["status"] for s in stats] == [L.OK] * B, stats
    L.call("hfm_device_timeouts", C.byref(cnt), 0)
    assert cnt.value == 0
    for i in range(B):
        oop = mg.Sigma7(sig[0, i], sig[1, i], sig[2, i], dtype=np.float64)
        assert mg.rel_residual(oop, phi[i].double().cpu().numpy(), f[i]) < 2e-6
