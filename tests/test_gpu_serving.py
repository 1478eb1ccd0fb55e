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


def test_native_server_same_bits_as_python_server(hfm, S):
    """The C-ABI serving loop (hfm_serve_*) over the same buckets gives every request the
    Python server's float64 solution bit for bit, and reaches the tolerance."""
    sv, torch = S
    edges = (16, 32)
    reqs = sv.make_stream(count=10, rate=1e6, edges=edges, log_std=(0.5, 2.0), seed=21)
    py = sv.SolveServer(edges=edges, slots=4, keep_solutions=True, cycles_per_tick=4)
    try:
        ref = {r.rid: r for r in py.serve(reqs, realtime=False)}
    finally:
        py.close()
    nat = sv.NativeServer(cfg=py.cfg, edges=edges, slots=4, cycles_per_tick=4)
    try:
        assert nat.bucket_slots(16) == 4 and nat.bucket_slots(32) == 4
        done, tickets = nat.serve(reqs)
        assert nat.pending() == (0, 0)
    finally:
        nat.close()
    for req, t in zip(reqs, tickets):
        d = done[t]
        assert d["status"] == 0, d
        assert (d["cycles"], d["outer"]) == (ref[req.rid].cycles, ref[req.rid].outer)
        np.testing.assert_array_equal(d["x"].cpu().numpy(), ref[req.rid].phi.cpu().numpy())
        assert _check_true_residual(req, d["x"], 1e-6) < 1e-6


def test_native_server_cancel(hfm, S):
    """A queued and a running request cancelled through hfm_serve_cancel are reported as
    HFM_ERR_CANCELLED; the others finish; a finished ticket cannot be cancelled."""
    sv, torch = S
    L = hfm._lib
    reqs = sv.make_stream(count=4, rate=1e6, edges=(32,), log_std=(1.0, 1.0), seed=23)
    nat = sv.NativeServer(edges=(32,), slots=2, cycles_per_tick=2)
    try:
        t = [nat.submit(r) for r in reqs]
        done = {d["ticket"]: d for d in nat.poll()}   # admits two, launches
        nat.cancel(t[3])                              # still queued
        nat.cancel(t[0])                              # running
        while len(done) < 4:
            for d in nat.poll():
                done[d["ticket"]] = d
        with pytest.raises(L.HfmError):
            nat.cancel(t[1])
    finally:
        nat.close()
    assert done[t[0]]["status"] == L.ERR_CANCELLED and done[t[3]]["status"] == L.ERR_CANCELLED
    assert done[t[1]]["status"] == 0 and done[t[2]]["status"] == 0
