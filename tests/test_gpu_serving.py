"""Continuous-batching server: every request reaches the tolerance, the result is the same
alone and in the mix (within the tolerance), and admission respects the HBM budget."""
import numpy as np
import pytest

from oracle import mg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def S(hfm):
    import torch
    return hfm.serving, torch


def _check_true_residual(req, phi, tol):
    sig = req.sigma.double().cpu().numpy()
    f = req.rhs.double().cpu().numpy()
    op = mg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float64)
    return mg.rel_residual(op, phi.double().cpu().numpy(), f)


def test_stream_same_alone_and_in_mix(hfm, S):
    sv, torch = S
    reqs = sv.make_stream(count=24, rate=4000.0, edges=(16, 24, 32), log_std=(0.5, 2.0), seed=5)
    server = sv.SolveServer(edges=(16, 24, 32), slots=4, keep_solutions=True, cycles_per_tick=2)
    try:
        res = server.serve(reqs, realtime=True)
    finally:
        server.close()
    assert len(res) == 24
    by_id = {r.rid: r for r in res}
    alone, _ = sv.solve_one_at_a_time(reqs, cfg=server.cfg, keep_solutions=True)
    for req in reqs:
        r = by_id[req.rid]
        assert r.status == 0, r
        assert _check_true_residual(req, r.phi, 1e-6) < 1e-6
        a = [x for x in alone if x.rid == req.rid][0]
        assert a.status == 0
        # same request alone (one-slot handle) and in the mix: both 1e-6 solutions of the same
        # system; they agree to the accuracy the tolerance allows
        d = (r.phi - a.phi).norm() / a.phi.norm()
        assert float(d) < 1e-4, float(d)
        assert r.latency > 0


def test_budget_limits_slots_and_queues(hfm, S):
    sv, torch = S
    per = hfm.multigrid.footprint_bytes(hfm.multigrid.SolverConfig(accel="ir", storage="bf16"),
                                        hfm._lib.OP_SIGMA7, (32, 32, 32), 1)
    budget = per * 3 + 1  # room for three 32^3 slots in total
    server = sv.SolveServer(edges=(32,), slots=8, budget_bytes=budget)
    try:
        assert server.buckets[32].slots == 2  # 8 -> 4 -> 2
        reqs = sv.make_stream(count=6, rate=1e6, edges=(32,), log_std=(1.0, 1.0), seed=9)
        res = server.serve(reqs, realtime=False)
    finally:
        server.close()
    assert sorted(r.rid for r in res) == list(range(6))
    assert all(r.status == 0 for r in res)
    # with two slots, later requests waited: admission time after arrival
    assert max(r.admitted - reqs[r.rid].arrival for r in res) > 0
