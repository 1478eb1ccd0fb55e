"""Z-slab decomposition on the GPU with the library's kernels.

All slabs run in one process here (``LocalSlabs``: the halo update is a plane copy).  Two GPUs
talking over NCCL use the same solver with ``DistSlabs``, which the CPU suite runs as two gloo
ranks.  Checked here:

* ``hfm_dot_f64`` and the CG vector updates against float64 torch arithmetic;
* one V-cycle gives the same bits over 1, 2 and 4 slabs, with agglomerated or distributed
  coarse levels, for the variable-coefficient, constant 7-point and 27-point operators, and
  agrees with the float32 oracle's one-domain V-cycle to 1e-5 of the field's largest value;
* PCG over 4 slabs takes the iterations of the one-slab solve, gives the same bits eagerly and
  as a replayed CUDA graph, and reaches the tolerance on the whole grid (residual recomputed with the float64 oracle operator); the one-GPU handle
  (``hfm_mg_solve``, same cycle) lands within one iteration and 1e-3 of the same solution.
"""
import ctypes as C
import datetime
import os
import socket
import sys

import numpy as np
import pytest

from oracle import mg as M, weights as OW

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def T(hfm):
    import torch
    return torch


def _kind_op(hfm, kind, sig_slabs=None):
    if kind == "sigma7":
        return hfm.slab.SlabSigma7(*sig_slabs, c=(1.0, 1.0, 1.0))
    if kind == "const7":
        return hfm.ops.Const7(0.5, 1.0, 2.0)
    return hfm.ops.Stencil27(OW.w5_pressure27())


def _oracle_op(kind, sig):
    if kind == "sigma7":
        return M.Sigma7(*sig, c=(1.0, 1.0, 1.0))
    if kind == "const7":
        return M.const7(0.5, 1.0, 2.0)
    return M.Stencil27(OW.w5_pressure27())


def _make(hfm, T, kind, shape, world, agg, cfg, sig):
    S = hfm.slab
    grp = S.LocalSlabs(world)
    ss = None
    if kind == "sigma7":
        ss = [S.split(T.from_numpy(a).cuda(), grp) for a in sig]
    return S.SlabMultigrid(shape, _kind_op(hfm, kind, ss), cfg, group=grp,
                           agglomerate_cells=agg), grp


@pytest.mark.parametrize("n,B,off", [(4096, 1, 0), (1000, 3, 0), (4097, 2, 1)])
def test_dot_and_cg_updates(hfm, T, n, B, off):
    L = hfm._lib
    stride = n + 24 + off
    g = T.Generator(device="cuda").manual_seed(3)
    buf = [T.randn(B * stride + 8, device="cuda", generator=g) for _ in range(5)]
    x, r, p, q, z = (a[off:] for a in buf)
    view = lambda a: a[:B * stride].view(B, stride)[:, :n]
    scratch = T.empty(max(8, L.lib().hfm_reduce_scratch_bytes(n, B)), dtype=T.uint8, device="cuda")
    out = T.empty(B, dtype=T.float64, device="cuda")
    s = C.c_void_p(T.cuda.current_stream().cuda_stream)
    P = lambda a: C.c_void_p(a.data_ptr())
    L.call("hfm_dot_f64", P(x), P(r), n, B, stride, P(out), P(scratch), s)
    ref = (view(x).double() * view(r).double()).sum(1)
    assert T.allclose(out, ref, rtol=1e-12, atol=1e-12)
    num = T.tensor([2.5], dtype=T.float64, device="cuda")
    den = T.tensor([-0.75], dtype=T.float64, device="cuda")
    a = np.float32(2.5 / -0.75)
    x0, r0, p0, q0, z0 = (view(t).clone() for t in (x, r, p, q, z))
    whole = [t.clone() for t in buf]
    L.call("hfm_cg_update_xr", P(x), P(r), P(p), P(q), P(num), P(den), n, B, stride, s)
    assert T.allclose(view(x), x0 + float(a) * p0, rtol=1e-6, atol=1e-6)
    assert T.allclose(view(r), r0 - float(a) * q0, rtol=1e-6, atol=1e-6)
    # cells outside the instances (the halo planes of a slab) are untouched
    for k in (0, 1):
        keep = T.ones_like(buf[k], dtype=T.bool)
        keep[off:][:B * stride].view(B, stride)[:, :n] = False
        assert T.equal(buf[k][keep], whole[k][keep])
    L.call("hfm_cg_update_p", P(p), P(z), P(num), P(den), n, B, stride, s)
    assert T.allclose(view(p), z0 + float(a) * p0, rtol=1e-6, atol=1e-6)
    view(p).fill_(float("nan"))
    L.call("hfm_cg_update_p", P(p), P(z), C.c_void_p(0), C.c_void_p(0), n, B, stride, s)
    assert T.equal(view(p), z0)        # first iteration: p = z, stale contents ignored


@pytest.mark.parametrize("kind", ["sigma7", "const7", "k27"])
def test_vcycle_same_bits_for_any_slab_count(hfm, T, kind):
    M_ = hfm.multigrid
    shape = (64, 64, 64)
    rng = np.random.default_rng(1)
    sig = hfm.problems.anisotropic_sigma(shape, 2, 1.0) if kind == "sigma7" else None
    b = rng.standard_normal(shape).astype(np.float32)
    phi = rng.standard_normal(shape).astype(np.float32)
    cfg = M_.SolverConfig(accel="cg")
    outs = {}
    for world, agg in ((1, 0), (2, 0), (4, 0), (2, 32 ** 3), (4, 32 ** 3), (4, 8 ** 3)):
        mg, grp = _make(hfm, T, kind, shape, world, agg, cfg, sig)
        S = hfm.slab
        v = mg.vcycle(S.split(T.from_numpy(phi).cuda(), grp), S.split(T.from_numpy(b).cuda(), grp))
        outs[(world, agg)] = v.reshape(shape).cpu().numpy()
    ref = outs[(1, 0)]
    for k, v in outs.items():
        np.testing.assert_array_equal(v, ref, err_msg=str(k))


@pytest.mark.parametrize("kind", ["sigma7", "const7", "k27"])
def test_vcycle_matches_oracle(hfm, T, kind):
    shape = (32, 48, 48)
    rng = np.random.default_rng(2)
    sig = hfm.problems.anisotropic_sigma(shape, 3, 1.0) if kind == "sigma7" else None
    b = rng.standard_normal(shape).astype(np.float32)
    phi = rng.standard_normal(shape).astype(np.float32)
    cfg = hfm.multigrid.SolverConfig(accel="cg")
    mg, grp = _make(hfm, T, kind, shape, 4, 0, cfg, sig)
    S = hfm.slab
    v = mg.vcycle(S.split(T.from_numpy(phi).cuda(), grp), S.split(T.from_numpy(b).cuda(), grp))
    op = _oracle_op(kind, sig)
    ops = M.hierarchy(op, len(S.level_shapes(shape, 0, cfg.min_coarse_edge)), cfg.coarse_scale)
    ref = M.vcycle(ops, 0, phi, b, M.CycleConfig())
    got = v.reshape(shape).cpu().numpy()
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 1e-5, err


def test_pcg_over_slabs(hfm, T):
    P = hfm.problems
    n = 64
    shape = (n, n, n)
    sig = P.anisotropic_sigma(shape, 5, 1.0)
    f = P.dipole(shape, 5)
    cfg = hfm.multigrid.SolverConfig(accel="cg", tol=1e-6)
    res = {}
    for world in (1, 4):
        mg, grp = _make(hfm, T, "sigma7", shape, world, 32 ** 3, cfg, sig)
        x, st = mg.solve(hfm.slab.split(T.from_numpy(f).cuda(), grp))
        assert st["converged"], st
        res[world] = (x.reshape(shape).cpu().numpy(), st)
    assert res[1][1]["iterations"] == res[4][1]["iterations"]
    x4 = res[4][0]
    # the captured CG iteration replays the eager kernels: same bits, also on a second solve
    mg, grp = _make(hfm, T, "sigma7", shape, 4, 32 ** 3, cfg, sig)
    mg.graphs = False
    xe, ste = mg.solve(hfm.slab.split(T.from_numpy(f).cuda(), grp))
    assert ste["history"] == res[4][1]["history"]
    np.testing.assert_array_equal(xe.reshape(shape).cpu().numpy(), x4)
    mg.graphs = True
    for _ in range(2):
        xg, stg = mg.solve(hfm.slab.split(T.from_numpy(f).cuda(), grp))
        np.testing.assert_array_equal(xg.reshape(shape).cpu().numpy(), x4)
    np.testing.assert_allclose(x4, res[1][0], rtol=0, atol=1e-5 * np.abs(x4).max())
    oop = M.Sigma7(*sig, dtype=np.float64)
    assert M.rel_residual(oop, x4.astype(np.float64), f) < 1.5e-6
    # the one-GPU handle on the same system and cycle
    Mg = hfm.multigrid
    with Mg.Multigrid(shape, hfm._lib.OP_SIGMA7, cfg, slots=1) as h:
        h.set_operator(hfm.ops.Sigma7(*(T.from_numpy(sig[k]).cuda() for k in range(3))))
        phi, st = h.solve(T.from_numpy(f[None]).cuda())
    assert abs(st[0]["cycles"] - res[4][1]["iterations"]) <= 1, (st, res[4][1]["iterations"])
    ph = phi[0].cpu().numpy()
    assert np.abs(ph - x4).max() / np.abs(ph).max() < 1e-3


def test_stationary_cycles_over_slabs(hfm, T):
    P = hfm.problems
    shape = (64, 48, 48)
    sig = P.anisotropic_sigma(shape, 6, 0.5)
    f = P.dipole(shape, 6)
    cfg = hfm.multigrid.SolverConfig(accel="none", tol=1e-6, max_cycles=200)
    out = {}
    for world in (1, 2):
        mg, grp = _make(hfm, T, "sigma7", shape, world, 0, cfg, sig)
        x, st = mg.solve(hfm.slab.split(T.from_numpy(f).cuda(), grp))
        assert st["converged"], st
        out[world] = (x.reshape(shape).cpu().numpy(), st["iterations"])
    assert out[1][1] == out[2][1]
    np.testing.assert_array_equal(out[1][0], out[2][0])


def _nccl_rank(port, q):
    ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    import __graft_entry__ as ge
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        hfm = ge.load_package()
        S, P = hfm.slab, hfm.problems
        shape = (64, 64, 64)
        sig = [torch.from_numpy(a).cuda() for a in P.anisotropic_sigma(shape, 8, 1.0)]
        f = torch.from_numpy(P.dipole(shape, 8)).cuda()
        cfg = hfm.multigrid.SolverConfig(accel="cg", tol=1e-6)
        out = []
        for grp in (S.DistSlabs(), S.LocalSlabs(1)):
            mg = S.SlabMultigrid(shape, S.SlabSigma7(*(S.split(a, grp) for a in sig)), cfg,
                                 group=grp, agglomerate_cells=16 ** 3)
            x, st = mg.solve(S.split(f, grp))
            out.append((x.cpu().numpy(), st["history"], mg.graphs))
        q.put(out)
    finally:
        dist.destroy_process_group()


def test_nccl_group_of_one_equals_local(hfm):
    """``DistSlabs`` on an NCCL group of one rank (all-gather of the coarse levels and the dot
    all-reduces through NCCL, eager) gives the bits of ``LocalSlabs(1)`` (graph replay).  A
    single rank has no halo partner; the send / recv path runs in the CPU suite on gloo."""
    import torch.multiprocessing as mp
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_rank, args=(port, q))
    p.start()
    (xd, hd, gd), (xl, hl, gl) = q.get(timeout=300)
    p.join(timeout=60)
    assert p.exitcode == 0
    assert not gd and gl
    assert hd == hl
    np.testing.assert_array_equal(xd, xl)
