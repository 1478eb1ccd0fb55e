"""Z-slab decomposition of one solve, host logic on the CPU.

The slab solver runs with the oracle's float32 operators as its kernel set
(``tests/_slab_oracle.py``), so halo planes, wall planes, the level plan, agglomeration and
conjugate gradients over slabs are checked without a GPU:

* one V-cycle over 1, 2 and 4 slabs equals the oracle's one-domain V-cycle bit for bit, for
  every way of splitting the hierarchy into distributed and agglomerated levels;
* preconditioned CG and stationary cycles take the oracle's iteration count and agree with its
  solution to 1e-5 of the largest value (dot products are summed per slab, so the last bits
  differ);
* two and four gloo ranks (``DistSlabs``, halo planes by send / recv, coarse levels by
  all-gather) give the same bits as one process; with four, the middle ranks exchange with
  both neighbours;
* two subgroups of two ranks each solve their own problem side by side (halo peers are the
  subgroup's global ranks).
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch

from oracle import mg as M, weights as OW

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HERE = os.path.dirname(os.path.abspath(__file__))
SHAPE = (32, 16, 16)


def _pkg():
    import __graft_entry__ as ge
    return ge.load_package()


def _problem(kind, seed=0, shape=SHAPE):
    rng = np.random.default_rng(seed)
    b = rng.standard_normal(shape).astype(np.float32)
    phi0 = rng.standard_normal(shape).astype(np.float32)
    sig = None
    if kind == "sigma7":
        sig = [np.exp(0.7 * rng.standard_normal(shape)).astype(np.float32) for _ in range(3)]
        op = M.Sigma7(*sig, c=(1.0, 1.0, 1.0))
    elif kind == "const7":
        op = M.const7(0.5, 1.0, 2.0)
    else:
        op = M.Stencil27(OW.w5_pressure27())
    return b, phi0, sig, op


def _slab_op(pkg, kind, sig, group):
    S = pkg.slab
    if kind == "sigma7":
        return S.SlabSigma7(*(S.split(torch.from_numpy(a), group) for a in sig), c=(1.0, 1.0, 1.0))
    if kind == "const7":
        return pkg.ops.Const7(0.5, 1.0, 2.0)
    return pkg.ops.Stencil27(OW.w5_pressure27())


def _cfgs(pkg, accel="cg"):
    cfg = pkg.multigrid.SolverConfig(accel=accel, min_coarse_edge=2, coarse_sweeps=8)
    ocfg = M.CycleConfig(nu_pre=2, nu_post=2, omega=2.0 / 3.0, coarse_sweeps=8)
    return cfg, ocfg


def _oracle_ops(op, pkg, cfg):
    n = len(pkg.slab.level_shapes(SHAPE, cfg.n_levels, cfg.min_coarse_edge))
    return M.hierarchy(op, n, cfg.coarse_scale)


def _solver(pkg, kind, sig, world, agg, cfg):
    from _slab_oracle import OracleSlabKernels
    S = pkg.slab
    grp = S.LocalSlabs(world)
    return S.SlabMultigrid(SHAPE, _slab_op(pkg, kind, sig, grp), cfg, group=grp, device="cpu",
                           agglomerate_cells=agg, kernels=OracleSlabKernels()), grp


def test_level_plan():
    pkg = _pkg()
    cfg, _ = _cfgs(pkg)
    _, _, sig, _ = _problem("const7")
    # (32,16,16) -> (16,8,8) -> (8,4,4) -> (4,2,2)
    for world, agg, la in ((1, 0, 4), (4, 0, 4), (4, 32 ** 3, 1), (2, 200, 2), (4, 600, 2)):
        mg, _ = _solver(pkg, "const7", sig, world, agg, cfg)
        assert mg.la == la, (world, agg, mg.la)
    with pytest.raises(ValueError):
        _solver(pkg, "const7", sig, 3, 0, cfg)       # 32 planes over 3 slabs
    with pytest.raises(ValueError):
        _solver(pkg, "const7", sig, 32, 0, cfg)      # one plane a slab cannot halve


@pytest.mark.parametrize("kind", ["sigma7", "const7", "k27"])
@pytest.mark.parametrize("world,agg", [(1, 0), (2, 0), (4, 0), (2, 32 ** 3), (4, 600)])
def test_vcycle_bitwise_equals_one_domain_oracle(kind, world, agg):
    pkg = _pkg()
    cfg, ocfg = _cfgs(pkg)
    b, phi0, sig, op = _problem(kind, seed=world)
    mg, grp = _solver(pkg, kind, sig, world, agg, cfg)
    S = pkg.slab
    out = mg.vcycle(S.split(torch.from_numpy(phi0), grp), S.split(torch.from_numpy(b), grp))
    ref = M.vcycle(_oracle_ops(op, pkg, cfg), 0, phi0, b, ocfg)
    np.testing.assert_array_equal(out.reshape(SHAPE).numpy(), ref)
    # zero initial guess too (the preconditioner form)
    out = mg.vcycle(None, S.split(torch.from_numpy(b), grp))
    ref = M.vcycle(_oracle_ops(op, pkg, cfg), 0, np.zeros_like(b), b, ocfg)
    np.testing.assert_array_equal(out.reshape(SHAPE).numpy(), ref)


@pytest.mark.parametrize("kind", ["sigma7", "k27"])
@pytest.mark.parametrize("world,agg", [(1, 0), (4, 600)])
def test_pcg_and_stationary_match_oracle(kind, world, agg):
    pkg = _pkg()
    S = pkg.slab
    b, _, sig, op = _problem(kind, seed=10 + world)
    cfg, ocfg = _cfgs(pkg, "cg")
    mg, grp = _solver(pkg, kind, sig, world, agg, cfg)
    x, st = mg.solve(S.split(torch.from_numpy(b), grp))
    xr, hist = M.pcg_solve(_oracle_ops(op, pkg, cfg), b, ocfg, tol=cfg.tol)
    assert st["converged"] and st["iterations"] == len(hist) - 1
    assert st["rel_resid"] == pytest.approx(hist[-1], rel=1e-3)
    err = np.abs(x.reshape(SHAPE).numpy() - xr).max() / np.abs(xr).max()
    assert err < 1e-5, err

    cfg, ocfg = _cfgs(pkg, "none")
    mg, grp = _solver(pkg, kind, sig, world, agg, cfg)
    x, st = mg.solve(S.split(torch.from_numpy(b), grp))
    xr, hist = M.solve(_oracle_ops(op, pkg, cfg), b, ocfg, tol=cfg.tol)
    assert st["converged"] and st["iterations"] == len(hist) - 1
    err = np.abs(x.reshape(SHAPE).numpy() - xr).max() / np.abs(xr).max()
    assert err < 1e-5, err


# ------------------------------------------------------------------------------ gloo ranks
def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, agg, q):
    sys.path[:0] = [ROOT, HERE]
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from _slab_oracle import OracleSlabKernels
        pkg = _pkg()
        S = pkg.slab
        grp = S.DistSlabs()
        cfg, _ = _cfgs(pkg, "cg")
        b, phi0, sig, _ = _problem("sigma7", seed=7)
        mg = S.SlabMultigrid(SHAPE, _slab_op(pkg, "sigma7", sig, grp), cfg, group=grp,
                             device="cpu", agglomerate_cells=agg, kernels=OracleSlabKernels())
        v = mg.vcycle(S.split(torch.from_numpy(phi0), grp), S.split(torch.from_numpy(b), grp))
        x, st = mg.solve(S.split(torch.from_numpy(b), grp))
        q.put((rank, mg.la, v.numpy(), x.numpy(), st["iterations"], st["history"]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,agg", [(2, 0), (2, 600), (4, 0), (4, 600)])
def test_gloo_ranks_equal_one_process(world, agg):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, agg, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=240) for _ in range(world)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    pkg = _pkg()
    cfg, ocfg = _cfgs(pkg, "cg")
    b, phi0, sig, op = _problem("sigma7", seed=7)
    assert {o[1] for o in out} == {4 if agg == 0 else 2}
    v = np.concatenate([o[2] for o in out]).reshape(SHAPE)
    np.testing.assert_array_equal(v, M.vcycle(_oracle_ops(op, pkg, cfg), 0, phi0, b, ocfg))
    mg, grp = _solver(pkg, "sigma7", sig, world, agg, cfg)
    x1, st1 = mg.solve(pkg.slab.split(torch.from_numpy(b), grp))
    x = np.concatenate([o[3] for o in out])
    assert {o[4] for o in out} == {st1["iterations"]}
    assert all(o[5] == out[0][5] for o in out)     # every rank saw the same residuals
    np.testing.assert_allclose(x, x1.numpy(), rtol=0, atol=1e-6 * np.abs(x).max())


def _subgroup_main(rank, port, q):
    """Four gloo ranks as two independent 2-slab solves on subgroups {0, 1} and {2, 3}: the
    halo peers are global ranks of the subgroup, and each pair solves its own problem."""
    sys.path[:0] = [ROOT, HERE]
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=4,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from _slab_oracle import OracleSlabKernels
        groups = [dist.new_group([0, 1]), dist.new_group([2, 3])]
        pkg = _pkg()
        S = pkg.slab
        grp = S.DistSlabs(groups[rank // 2])
        cfg, _ = _cfgs(pkg, "cg")
        b, _, sig, _ = _problem("sigma7", seed=20 + rank // 2)
        mg = S.SlabMultigrid(SHAPE, _slab_op(pkg, "sigma7", sig, grp), cfg, group=grp,
                             device="cpu", agglomerate_cells=600, kernels=OracleSlabKernels())
        x, st = mg.solve(S.split(torch.from_numpy(b), grp))
        q.put((rank, grp.rank, grp.world, x.numpy(), st["iterations"]))
    finally:
        dist.destroy_process_group()


def test_gloo_subgroups_solve_independently():
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_subgroup_main, args=(r, port, q)) for r in range(4)]
    for p in procs:
        p.start()
    out = sorted([q.get(timeout=240) for _ in range(4)], key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [(o[1], o[2]) for o in out] == [(0, 2), (1, 2), (0, 2), (1, 2)]
    pkg = _pkg()
    cfg, _ = _cfgs(pkg, "cg")
    for pair in (0, 1):
        b, _, sig, _ = _problem("sigma7", seed=20 + pair)
        mg, grp = _solver(pkg, "sigma7", sig, 2, 600, cfg)
        x1, st1 = mg.solve(pkg.slab.split(torch.from_numpy(b), grp))
        mine = out[2 * pair:2 * pair + 2]
        assert {o[4] for o in mine} == {st1["iterations"]}
        x = np.concatenate([o[3] for o in mine])
        np.testing.assert_allclose(x, x1.numpy(), rtol=0, atol=1e-6 * np.abs(x).max())
