"""NS time-stepper operators on the GPU against the oracle, and a full
reference time step."""
import os

import numpy as np
import pytest

from oracle import ns as ons

pytestmark = pytest.mark.gpu
SHAPE = (10, 12, 14)


def close(got, ref, rtol=1e-5):
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    err = np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-30)
    assert err <= rtol, "max rel err %.3e > %.1e" % (err, rtol)


@pytest.fixture(scope="module")
def env(hfm):
    import torch
    rng = np.random.default_rng(31)
    f = {k: rng.standard_normal(SHAPE).astype(np.float32) for k in ("u", "v", "w", "p", "b")}
    return hfm, torch, f


def D(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def test_boundary_conditions(env):
    hfm, torch, f = env
    ns = hfm.ns
    u, v, w = D(torch, f["u"]), D(torch, f["v"]), D(torch, f["w"])
    ns.boundary_condition_velocity(u, v, w, 1.5)
    ru, rv, rw = ons.bc_velocity(f["u"], f["v"], f["w"], 1.5)
    np.testing.assert_array_equal(u.cpu().numpy(), ru)
    np.testing.assert_array_equal(v.cpu().numpy(), rv)
    np.testing.assert_array_equal(w.cpu().numpy(), rw)
    p = D(torch, f["p"])
    ns.boundary_condition_pressure(p)
    np.testing.assert_array_equal(p.cpu().numpy(), ons.bc_pressure(f["p"]))


def test_momentum_gradient_divergence_ibm(env):
    hfm, torch, f = env
    ns, W = hfm.ns, hfm.weights
    dt = 0.1
    Kd = W.diffusion27(dt, 0.25)
    Kx, Ky, Kz = W.advection(dt)
    u, v, w = (D(torch, f[k]) for k in "uvw")
    ou, ov, ow = (torch.empty_like(u) for _ in range(3))
    ns.momentum_stage((u, v, w), (u, v, w), (ou, ov, ow), Kd, Kx, Ky, Kz, 0.5)
    for got, name in zip((ou, ov, ow), "uvw"):
        ref = 0.5 * ons.momentum_rhs(f[name], f["u"], f["v"], f["w"], Kd, Kx, Ky, Kz) + f[name]
        close(got.cpu(), ref)
    p = D(torch, f["p"])
    u2, v2, w2 = (D(torch, f[k]) for k in "uvw")
    ns.pressure_gradient(p, u2, v2, w2, Kx, Ky, Kz)
    for got, ref in zip((u2, v2, w2), ons.pressure_gradient(f["p"], f["u"], f["v"], f["w"], Kx, Ky, Kz)):
        close(got.cpu(), ref)
    Su, Sv, Sw = W.divergence(dt)
    b = torch.empty_like(u)
    ns.divergence(u, v, w, b, Su, Sv, Sw, bc_source=True)
    close(b.cpu(), ons.divergence_rhs(f["u"], f["v"], f["w"], Su, Sv, Sw))
    sig = np.where(np.random.default_rng(2).random(SHAPE) < 0.2, 1e5, 0).astype(np.float32)
    u3, v3, w3 = (D(torch, f[k]) for k in "uvw")
    ns.bluff_body(u3, v3, w3, D(torch, sig), dt)
    for got, ref in zip((u3, v3, w3), ons.bluff_body(f["u"], f["v"], f["w"], sig, dt)):
        np.testing.assert_allclose(got.cpu().numpy(), ref, rtol=1e-6, atol=1e-12)


@pytest.mark.parametrize("multi_itr", [2, 5])
def test_reference_step(env, multi_itr):
    """Two reference time steps (naiver_stokes_3D.py:571-727) on 16^3 with an obstacle."""
    hfm, torch, f = env
    ns = hfm.ns
    n = 16
    cfg = ns.NSConfig(dt=0.1, Re=0.25, ub=1.0, pressure="reference", multi_itr=multi_itr)
    sig = ns.obstacle_mask((n, n, n), n_boxes=2, footprint=(2, 4), height=(3, 6), seed=1)
    st = ns.NSStepper((n, n, n), cfg, sigma=sig)
    W = hfm.weights
    Kd = W.diffusion27(cfg.dt, cfg.Re)
    Kx, Ky, Kz = W.advection(cfg.dt)
    Su, Sv, Sw = W.divergence(cfg.dt)
    Kp = W.pressure27()
    z = np.zeros((n, n, n), np.float32)
    ru, rv, rw, rp = z, z, z, z
    signp = sig.cpu().numpy()
    try:
        for _ in range(2):
            st.step()
            ru, rv, rw, rp = ons.step(ru, rv, rw, rp, signp, cfg.dt, cfg.ub, Kd, Kx, Ky, Kz, Su, Sv,
                                      Sw, Kp, 4, multi_itr)
        for got, ref in zip((st.u, st.v, st.w, st.p), (ru, rv, rw, rp)):
            close(got.cpu(), ref, rtol=1e-4)
    finally:
        st.close()


def test_petrov_galerkin_dissipation_and_momentum(env):
    """INHALE_demo.ipynb cells 20 and 24: the Petrov-Galerkin terms (with an immersed body)
    and the momentum update that uses them, against the oracle."""
    hfm, torch, f = env
    ns, W = hfm.ns, hfm.weights
    dt = 0.5
    Kd = W.diffusion27(dt, 1.0 / 20.0)
    Kx, Ky, Kz = W.advection(dt, factor=0.5)
    sig = np.where(np.random.default_rng(7).random(SHAPE) < 0.1, 1e5, 0).astype(np.float32)
    u, v, w = (D(torch, f[k]) for k in "uvw")
    k = tuple(torch.empty_like(u) for _ in range(3))
    ns.pg_dissipation(u, v, w, D(torch, sig), k, Kd, Kx, Ky, Kz, dt, 1e-3)
    refs = ons.pg_dissipation(f["u"], f["v"], f["w"], sig, dt, 1e-3, Kd, Kx, Ky, Kz)
    for got, ref in zip(k, refs):
        close(got.cpu(), ref, rtol=1e-4)
    cfg = ns.NSConfig(dt=dt, Re=1.0 / 20.0, adv_factor=0.5, pg=True, pressure="reference",
                      multi_itr=2)
    st = ns.NSStepper(SHAPE, cfg, sigma=D(torch, sig))
    for name in "uvw":
        getattr(st, name).copy_(D(torch, f[name]))
    b = (st.bu, st.bv, st.bw)
    n = (st.nu, st.nv, st.nw)
    kk = (st.kx, st.ky, st.kz)
    ns.pg_dissipation(st.u, st.v, st.w, st.sigma, kk, st.Kdif, st.Kx, st.Ky, st.Kz, dt)
    ns.momentum_stage_pg((st.u, st.v, st.w), (st.u, st.v, st.w), b, kk, st.Kx, st.Ky, st.Kz, 0.5)
    ns.boundary_condition_velocity(*b, cfg.ub)
    ns.pg_dissipation(*b, st.sigma, kk, st.Kdif, st.Kx, st.Ky, st.Kz, dt)
    ns.momentum_stage_pg(b, (st.u, st.v, st.w), n, kk, st.Kx, st.Ky, st.Kz, 1.0)
    refs = ons.momentum_pg(f["u"], f["v"], f["w"], cfg.ub, sig, dt, 1e-3, Kd, Kx, Ky, Kz)
    for got, ref in zip(n, refs):
        close(got.cpu(), ref, rtol=1e-4)
    st.close()
    # the stepper's own PG path, end to end on 16^3 with an obstacle
    s2 = ns.NSStepper((16, 16, 16), cfg, sigma=ns.obstacle_mask((16, 16, 16), n_boxes=2,
                                                                 footprint=(2, 4), height=(2, 6)))
    s2.u.fill_(1.0)
    for _ in range(3):
        s2.step()
    assert all(bool(torch.isfinite(t).all()) for t in (s2.u, s2.v, s2.w, s2.p))
    s2.close()


def test_checkpoint_restart_continues_bitwise(env, tmp_path):
    """N steps, save in the reference's .npy layout, a fresh stepper restarts from the files
    and takes N more: the fields equal those of 2N uninterrupted steps bit for bit, and the
    restart clock follows naiver_stokes_3D.py:531-549, 572 (ctime_old = nrestart dt, each step
    adds dt + ctime_old)."""
    hfm, torch, _ = env
    ns = hfm.ns
    shape, N = (16, 32, 32), 3
    cfg = ns.NSConfig(dt=0.5, dx=1.0, Re=0.05, ub=1.0, diffusion="7", pressure="fcycle", p_tol=1e-5)
    sig = ns.obstacle_mask(shape, n_boxes=4, footprint=(3, 6), height=(4, 10), sigma=1e5, seed=2)
    ref = ns.NSStepper(shape, cfg, sigma=sig)
    try:
        for _ in range(2 * N):
            ref.step()
        want = {k: getattr(ref, k).cpu().numpy() for k in ("u", "v", "w", "p")}
    finally:
        ref.close()
    a = ns.NSStepper(shape, cfg, sigma=sig)
    try:
        for _ in range(N):
            a.step()
        assert not a.save(str(tmp_path), n_out=2)  # step 3 is not a multiple of n_out = 2
        assert a.save(str(tmp_path), n_out=N)
        assert sorted(os.listdir(tmp_path)) == ["p3.npy", "u3.npy", "v3.npy", "w3.npy"]
        assert np.load(tmp_path / "u3.npy").shape == shape
    finally:
        a.close()
    b = ns.NSStepper(shape, cfg, sigma=sig)
    try:
        b.restart(str(tmp_path), N)
        assert b.itime == N and b.nrestart == N and b.ctime_old == N * cfg.dt
        for _ in range(N):
            b.step()
        assert b.itime == 2 * N
        # the reference's accumulation: ctime = ctime + dt + ctime_old at every step
        clock = 0.0
        for _ in range(N):
            clock = clock + cfg.dt + N * cfg.dt
        assert b.ctime == clock
        for k, v in want.items():
            np.testing.assert_array_equal(getattr(b, k).cpu().numpy(), v, err_msg=k)
        with pytest.raises(ValueError):
            np.save(tmp_path / "u9.npy", np.zeros((4, 4, 4), np.float32))
            for k in ("v", "w", "p"):
                np.save(tmp_path / ("%s9.npy" % k), np.zeros(shape, np.float32))
            b.restart(str(tmp_path), 9)
    finally:
        b.close()
