"""Every workload configuration at its own size, on the GPU, against the oracle.

One test per configuration (collected after the per-operator tests, so a failure here
leaves their results standing):

* obstacle flow, 64 x 128 x 128 with 24 boxes: three time steps of the stepper against the
  oracle's step with the same pressure stopping rule, every pressure solve reaching 1e-5;
* precision, 256^3 with sigma log-std 2: float64 refinement to 1e-10 around bf16 and fp16
  inner cycles, true residual recomputed by the float64 oracle operator, error against a
  float64 solve of the same system;
* Kolmogorov flow, 512^2: ten steps against the oracle's step;
* tomography, 96^3 with 32 sources x 64 receivers: the adjoint gradient against central
  finite differences (eps 1e-4) on 20 random cells;
* serving, edges {48, 96, 128} with 8 slots per bucket (TMA levels, the fused first two
  sweeps and the fused coarse cycle all engage): each request's float64 solution in the mix
  equals, bit for bit, the one it gets when served alone through the same bucket shape.
"""
import numpy as np
import pytest

from oracle import kolmogorov as K2
from oracle import mg as omg
from oracle import ns as ons

pytestmark = pytest.mark.gpu


def _rel_max(got, ref):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    return float(np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-30))


# ------------------------------------------------------------------ obstacle flow
def test_obstacle_flow_64x128x128_three_steps_match_oracle(hfm):
    """128 x 128 x 64 flow past 24 seeded boxes (dx 1, nu 0.05, dt 0.5, 7-point diffusion,
    F(2,2) pressure cycles to 1e-5 with the outflow rule): the GPU stepper against the
    oracle's time step (naiver_stokes_3D.py:571-727) for three steps, 1e-5 per field."""
    import torch
    ns, W = hfm.ns, hfm.weights
    shape = (64, 128, 128)
    cfg = ns.NSConfig(dt=0.5, dx=1.0, Re=0.05, ub=1.0, diffusion="7", pressure="fcycle", p_tol=1e-5)
    sig = ns.obstacle_mask(shape, n_boxes=24, footprint=(4, 16), height=(8, 40), sigma=1e5, seed=0)
    st = ns.NSStepper(shape, cfg, sigma=sig)
    try:
        levels = omg.level_shapes(shape)
        assert st.mg.levels == levels
        ops = omg.hierarchy(omg.Stencil27(st.Kp), len(levels), 0.5)
        ccfg = omg.CycleConfig(2, 2, 2.0 / 3.0, 32, zero_xend=True)
        oracle_cycles = []

        def pressure(p, b):
            p, cyc, rel = omg.cycle_to_tolerance(ops, p, b, ccfg, cfg.p_tol, 500, cycle="F")
            oracle_cycles.append(cyc)
            return p

        sigma = sig.cpu().numpy()
        z = np.zeros(shape, np.float32)
        ref = (z, z, z, z)
        for k in range(3):
            st.step()
            ref = ons.step(*ref, sigma, cfg.dt, cfg.ub, st.Kdif, st.Kx, st.Ky, st.Kz, st.Su,
                           st.Sv, st.Sw, st.Kp, 0, 0, pressure=pressure)
            assert st.p_status[-1] == 0 and st.p_rel[-1] < cfg.p_tol, (k, st.p_status, st.p_rel)
            assert st.p_cycles[-1] == oracle_cycles[-1], (st.p_cycles, oracle_cycles)
            torch.cuda.synchronize()
            for name, r in zip("uvwp", ref):
                err = _rel_max(getattr(st, name).cpu().numpy(), r)
                assert err <= 1e-5, (k, name, err)
        assert all(np.isfinite(a).all() for a in ref)
        assert float(st.u.abs().max()) > 0.5  # the inflow has entered the domain
    finally:
        st.close()


# ------------------------------------------------------------------ precision, 256^3
@pytest.fixture(scope="module")
def precision_problem(hfm):
    """256^3, sigma log-std 2 (contrast about 1e3), dipole source; the float64 reference
    solution is float64 refinement driven to 1e-13 (float32 inner cycles), whose own residual
    is checked by the float64 oracle operator."""
    import torch
    M, L, ops = hfm.multigrid, hfm._lib, hfm.ops
    n = 256
    sig = hfm.problems.anisotropic_sigma((n, n, n), seed=0, log_std=2.0)
    f = hfm.problems.dipole((n, n, n), seed=0).astype(np.float64)
    sd = torch.from_numpy(sig).cuda()
    fd = torch.from_numpy(f).cuda()
    op = ops.Sigma7(sd[0], sd[1], sd[2])

    def solve(storage, tol):
        cfg = M.SolverConfig(cycle="V", accel="ir", storage=storage, tol=tol, max_cycles=4000)
        with M.Multigrid((n, n, n), L.OP_SIGMA7, cfg, slots=1) as h:
            h.set_operator(op)
            h.load_f64(0, fd)
            for _ in range(1000):
                h.run(8)
                s = h.query()[0]
                if not s["active"]:
                    break
            return h.fetch_f64(0).cpu().numpy(), s

    op64 = omg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float64)
    x_ref, s_ref = solve("f32", 1e-13)
    assert s_ref["status"] == 0, s_ref
    assert omg.rel_residual(op64, x_ref, f) < 1e-12
    yield solve, op64, f, x_ref
    del sd, fd


@pytest.mark.parametrize("storage", ["bf16", "f16"])
def test_precision_256_refinement_to_1e10(hfm, precision_problem, storage):
    solve, op64, f, x_ref = precision_problem
    x, s = solve(storage, 1e-10)
    assert s["status"] == 0, (storage, s)
    rel = omg.rel_residual(op64, x, f)
    err = float(np.linalg.norm((x - x_ref).ravel()) / np.linalg.norm(x_ref.ravel()))
    print("precision 256^3 log-std 2, %s inner: %d inner iterations, %d refinement steps, "
          "true rel resid %.2e, error vs float64 solve %.2e" % (storage, s["cycles"], s["outer"], rel, err))
    assert rel < 1e-10, (storage, rel)
    assert abs(rel - s["rel_resid"]) <= 1e-3 * rel + 1e-14
    # the error is bounded by the condition number times the residual; measured ~1e-11
    assert err < 1e-8, (storage, err)


# ------------------------------------------------------------------ Kolmogorov, 512^2
def test_kolmogorov_512_ten_steps_match_oracle(hfm):
    """The doubly periodic Kolmogorov flow at 512^2 (nu 1/40, sin(4y) forcing, dt 1e-3, three
    pressure cycles per step): ten float32 GPU steps against ten float64 oracle steps."""
    KM = hfm.kolmogorov
    n = 512
    kf = KM.KolmogorovFlow(n=n, dt=1e-3, cycles=3, seed=0)
    u, v, p = (t.double().cpu().numpy() for t in (kf.u, kf.v, kf.p))
    om = K2.VCycle2D(K2.laplace5(kf.h), (n, n), dt=np.float64)
    for _ in range(10):
        kf.step()
        u, v, p = K2.ns_step(u, v, p, om, 3, kf.dt, kf.nu, kf.h)
    eu = _rel_max(kf.u.cpu().numpy(), u)
    ev = _rel_max(kf.v.cpu().numpy(), v)
    ep = _rel_max(kf.p.cpu().numpy(), p)
    print("kolmogorov 512^2, 10 steps: max rel err u %.2e v %.2e p %.2e" % (eu, ev, ep))
    assert eu <= 1e-5 and ev <= 1e-4 and ep <= 1e-3, (eu, ev, ep)


# ------------------------------------------------------------------ tomography, 96^3
def test_tomography_96_gradient_matches_finite_differences(hfm):
    """96^3, 32 dipole sources x 64 receivers on z = 0, data from the three-ellipsoid model,
    homogeneous start: the adjoint gradient w.r.t. log sigma_x, y, z against central finite
    differences of the misfit (eps 1e-4) on 20 random cells."""
    import torch
    tm = hfm.tomography
    n = 96
    survey = tm.make_survey(n=n, n_src=32, n_rec=64, seed=0)
    solver = tm.ForwardSolver(n, group=32, tol=1e-10)
    try:
        d_obs = tm.observe(tm.true_sigma(n, seed=0), survey, solver)
        logs = torch.zeros((3, n, n, n), dtype=torch.float64, device="cuda", requires_grad=True)
        tm.misfit(logs, survey, d_obs, solver).backward()
        g = logs.grad.cpu().numpy()
        gmax = np.abs(g).max()
        assert gmax > 0
        rng = np.random.default_rng(1)
        eps = 1e-4
        base = logs.detach().clone()
        worst = 0.0
        for _ in range(20):
            k, z, y, x = (int(rng.integers(0, 3)),) + tuple(int(v) for v in rng.integers(0, n, 3))
            lp, lm = base.clone(), base.clone()
            lp[k, z, y, x] += eps
            lm[k, z, y, x] -= eps
            fd = (tm.misfit_value(lp, survey, d_obs, solver) -
                  tm.misfit_value(lm, survey, d_obs, solver)) / (2 * eps)
            worst = max(worst, abs(fd - g[k, z, y, x]) / gmax)
            # float32 conductivities: exp(+-eps) is rounded to float32 (relative 6e-8 of a
            # 1e-4 step), so agreement is to about 1e-3 of the cell's own gradient
            assert abs(fd - g[k, z, y, x]) <= 2e-3 * abs(g[k, z, y, x]) + 1e-4 * gmax, \
                (k, z, y, x, fd, g[k, z, y, x])
        print("tomography 96^3 32x64: FD max error %.2e of max|g|" % worst)
    finally:
        solver.close()


# ------------------------------------------------------------------ serving, edges 48-128
def test_serving_48_96_128_same_bits_alone_and_in_mix(hfm):
    """A stream over edges {48, 96, 128} with 8 slots per bucket and bf16 inner cycles (so the
    TMA kernels, the fused first two pre-sweeps and the fused coarse cycle run): every
    request reaches 1e-6 (float64 oracle residual), and its float64 solution in the mix is
    bitwise the solution it gets served alone through a bucket of the same shape."""
    sv = hfm.serving
    edges = (48, 96, 128)
    reqs = sv.make_stream(count=30, rate=20000.0, edges=edges, log_std=(0.5, 2.0), seed=14)
    # more requests than slots per edge (9, 11, 10): every bucket fills up and some queue
    assert all(sum(r.n == e for r in reqs) > 8 for e in edges)
    server = sv.SolveServer(edges=edges, slots=8, keep_solutions=True, cycles_per_tick=4)
    try:
        assert all(b.slots == 8 for b in server.buckets.values())
        assert all(b.mg.levels[0][2] >= 48 for b in server.buckets.values())
        res = {r.rid: r for r in server.serve(reqs, realtime=True)}
    finally:
        server.close()
    assert sorted(res) == [r.rid for r in reqs]
    for e in edges:
        alone = sv.SolveServer(edges=(e,), slots=8, keep_solutions=True, cycles_per_tick=4)
        try:
            for req in (r for r in reqs if r.n == e):
                mix = res[req.rid]
                assert mix.status == 0, mix
                a = alone.serve([req], realtime=False)[0]
                assert a.status == 0 and a.cycles == mix.cycles and a.outer == mix.outer, (a, mix)
                np.testing.assert_array_equal(a.phi.cpu().numpy(), mix.phi.cpu().numpy())
                sig = req.sigma.double().cpu().numpy()
                op = omg.Sigma7(sig[0], sig[1], sig[2], dtype=np.float64)
                rel = omg.rel_residual(op, mix.phi.cpu().numpy(), req.rhs.double().cpu().numpy())
                assert rel < 1e-6, (req.rid, e, rel)
        finally:
            alone.close()
