"""The C-ABI library loads and exports every symbol include/hfm.h declares (no GPU calls)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hfm.h")


def declared_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(hfm_[a-z0-9_]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib(pkg):
    return pkg._lib.lib()


def test_header_declares_api():
    syms = declared_symbols()
    for must in ("hfm_conv3d_k3", "hfm_restrict_avg", "hfm_prolong_nearest", "hfm_op_jacobi",
                 "hfm_residual_restrict", "hfm_prolong_correct_smooth", "hfm_norm2_f64",
                 "hfm_mg_create", "hfm_mg_solve", "hfm_stencil7_var_jacobi",
                 "hfm_stencil27_residual"):
        assert must in syms


def test_every_declared_symbol_is_exported(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_header(pkg):
    assert set(declared_symbols()) == set(pkg._lib.SIGNATURES)


def test_host_only_calls(lib, pkg):
    L = pkg._lib
    assert lib.hfm_abi_version() == 1
    assert lib.hfm_status_string(L.ERR_NOT_CONVERGED) == b"HFM_ERR_NOT_CONVERGED"
    cfg = L.HfmMgConfig()
    lib.hfm_mg_config_default(C.byref(cfg))
    assert cfg.nu_pre == 2 and cfg.nu_post == 2 and abs(cfg.omega - 2 / 3) < 1e-7
    assert cfg.tol == 1e-6 and cfg.min_coarse_edge == 4
    f64 = lib.hfm_mg_footprint_bytes(C.byref(cfg), 64, 64, 64, 1)
    f128 = lib.hfm_mg_footprint_bytes(C.byref(cfg), 128, 128, 128, 1)
    assert 64 ** 3 * 24 < f64 < 64 ** 3 * 40
    assert 6 < f128 / f64 < 9
    assert lib.hfm_mg_footprint_bytes(C.byref(cfg), 64, 64, 64, 10) > 9 * f64
    assert lib.hfm_reduce_scratch_bytes(0, 1) == 0


def test_bad_arguments_fail_without_gpu(lib, pkg):
    """Argument validation happens on the host before any CUDA call."""
    L = pkg._lib
    st = lib.hfm_restrict_avg(None, None, 1, 4, 4, 4, None)
    assert st == L.ERR_BAD_ARG
    assert b"NULL" in lib.hfm_last_error()
    st = lib.hfm_conv3d_k3(None, None, 0, 4, 4, 4, None, None)
    assert st == L.ERR_BAD_ARG
    cfg = L.HfmMgConfig()
    lib.hfm_mg_config_default(C.byref(cfg))
    cfg.accel = L.ACCEL_CG
    cfg.nu_post = 1
    h = C.c_void_p()
    assert lib.hfm_mg_create(C.byref(cfg), 8, 8, 8, 1, C.byref(h)) == L.ERR_BAD_ARG
    assert b"symmetric" in lib.hfm_last_error()
    cfg.nu_post = 2
    cfg.cycle = L.CYCLE_F
    assert lib.hfm_mg_create(C.byref(cfg), 8, 8, 8, 1, C.byref(h)) == L.ERR_BAD_ARG
    assert b"F-cycle" in lib.hfm_last_error()


def test_slab_entry_points_validate_without_gpu(lib, pkg):
    """The Z-slab CG helpers reject bad pointers and strides on the host."""
    L = pkg._lib
    f = lib.hfm_dot_f64
    assert f(None, None, 16, 1, 16, None, None, None) == L.ERR_BAD_ARG
    buf = (C.c_float * 64)()
    out = (C.c_double * 2)()
    scratch = (C.c_char * 64)()
    # two instances whose stride is shorter than an instance overlap
    assert f(buf, buf, 32, 2, 16, out, scratch, None) == L.ERR_BAD_ARG
    assert b"hfm_dot_f64" in lib.hfm_last_error()
    d = (C.c_double * 1)()
    assert lib.hfm_cg_update_xr(buf, buf, buf, buf, None, d, 16, 1, 16, None) == L.ERR_BAD_ARG
    assert lib.hfm_cg_update_p(buf, buf, None, d, 16, 1, 16, None) == L.ERR_BAD_ARG
    assert lib.hfm_cg_update_p(buf, buf, d, d, 0, 1, 16, None) == L.ERR_BAD_ARG
    assert b"hfm_cg_update_p" in lib.hfm_last_error()


def test_reductions_reject_more_instances_than_grid_rows(lib, pkg):
    """One grid row per instance: B = 65536 is refused on the host with HFM_ERR_BAD_ARG, not
    left to fail as a launch error."""
    L = pkg._lib
    buf = (C.c_float * 64)()
    out = (C.c_double * 2)()
    scratch = (C.c_char * 64)()
    B = 65536
    assert lib.hfm_reduce_scratch_bytes(8, B) == 0
    assert lib.hfm_reduce_scratch_bytes(8, B - 1) > 0
    assert lib.hfm_norm2_f64(buf, 8, B, out, scratch, None) == L.ERR_BAD_ARG
    assert b"65535" in lib.hfm_last_error()
    assert lib.hfm_norm2_f64_noalloc(buf, 8, B, out, None) == L.ERR_BAD_ARG
    assert lib.hfm_dot_f64(buf, buf, 8, B, 8, out, scratch, None) == L.ERR_BAD_ARG
    assert lib.hfm_max_abs(buf, 8, B, buf, scratch, None) == L.ERR_BAD_ARG


def test_sawtooth_coarse_sweeps_option(pkg):
    """SolverConfig.reference(coarse_sweeps=k) sets the option bit only when k != 1, so the
    reference cycle's single coarsest sweep stays the default."""
    M, L = pkg.multigrid, pkg._lib
    one = M.SolverConfig.reference(n_levels=5).struct(L.OP_K27)
    assert not one.options & L.OPT_SAWTOOTH_COARSE_SWEEPS
    two = M.SolverConfig.reference(n_levels=5, coarse_sweeps=2).struct(L.OP_K27)
    assert two.options & L.OPT_SAWTOOTH_COARSE_SWEEPS and two.coarse_sweeps == 2
    v = M.SolverConfig(cycle="V", sawtooth_coarse_sweeps=3).struct(L.OP_SIGMA7)
    assert not v.options & L.OPT_SAWTOOTH_COARSE_SWEEPS and v.coarse_sweeps == 32


def test_face7_host_calls(lib, pkg):
    """FACE7 array sizes, argument checks of the face builder, and the handle footprint that
    counts the face arrays of 16-bit SIGMA7 levels (none with HFM_OPT_NO_FACES or float32)."""
    L = pkg._lib
    a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
    assert lib.hfm_face7_elems(4, 5, 6, C.byref(a), C.byref(b), C.byref(c)) == L.OK
    assert (a.value, b.value, c.value) == (4 * 5 * 14, 4 * 6 * 6, 5 * 5 * 6)
    assert lib.hfm_face7_elems(0, 5, 6, C.byref(a), C.byref(b), C.byref(c)) == L.ERR_BAD_ARG
    buf = (C.c_float * 64)()
    assert lib.hfm_sigma7_faces(L.BF16, None, buf, buf, 1.0, 1.0, 1.0, buf, buf, buf, 1, 2, 2, 2,
                                None) == L.ERR_BAD_ARG
    assert lib.hfm_sigma7_faces(L.F64, buf, buf, buf, 1.0, 1.0, 1.0, buf, buf, buf, 1, 2, 2, 2,
                                None) == L.ERR_BAD_ARG
    assert b"dtype" in lib.hfm_last_error()
    cfg = L.HfmMgConfig()
    lib.hfm_mg_config_default(C.byref(cfg))
    cfg.storage = L.BF16
    with_faces = lib.hfm_mg_footprint_bytes(C.byref(cfg), 128, 128, 128, 1)
    cfg.options = L.OPT_NO_FACES
    without = lib.hfm_mg_footprint_bytes(C.byref(cfg), 128, 128, 128, 1)
    # faces on the 128^3 and 64^3 levels (plane-marching kernels, X >= 48) and the 32^3 level
    # (register-queue kernels, more than 4096 cells): 3 arrays of about n cells, 2 bytes each
    extra = 2 * (128 * 128 * 136 + 128 * 129 * 128 + 129 * 128 * 128 +
                 64 * 64 * 72 + 64 * 65 * 64 + 65 * 64 * 64 +
                 32 * 32 * 40 + 32 * 33 * 32 + 33 * 32 * 32)
    assert with_faces - without == extra
    cfg.options = 0
    cfg.storage = L.F32
    f32 = lib.hfm_mg_footprint_bytes(C.byref(cfg), 128, 128, 128, 1)
    cfg.options = L.OPT_NO_FACES
    assert lib.hfm_mg_footprint_bytes(C.byref(cfg), 128, 128, 128, 1) == f32


def test_face7_smooth2_validates_without_gpu(lib, pkg):
    """The two-sweep entry point rejects null fields, aliasing, float32, other operator kinds
    and grids the kernel does not take before it touches the device."""
    L = pkg._lib
    buf = (C.c_float * 64)()
    addr = C.addressof(buf)
    al = C.c_void_p((addr + 15) & ~15)
    op = L.HfmOperator()
    op.kind, op.coef_dtype, op.scale = L.OP_FACE7, L.BF16, 1.0
    for i in range(3):
        op.coef[i] = al.value
    f = lambda *a: lib.hfm_face7_smooth2_typed(C.byref(op), *a)
    assert f(L.BF16, None, None, al, al, 1, 4, 16, 64, 0.6, None) == L.ERR_BAD_ARG
    assert f(L.BF16, al, None, al, al, 1, 4, 16, 64, 0.6, None) == L.ERR_BAD_ARG  # phi == out
    other = C.c_void_p(al.value + 16)
    assert f(L.BF16, al, None, al, other, 1, 4, 16, 40, 0.6, None) == L.ERR_UNSUPPORTED  # X < 48
    assert f(L.BF16, al, None, al, other, 1, 4, 8, 64, 0.6, None) == L.ERR_UNSUPPORTED   # Y < 16
    assert f(L.BF16, al, al, al, other, 1, 4, 16, 72, 0.6, None) == L.ERR_UNSUPPORTED    # X % 16
    op.coef_dtype = L.F32
    assert f(L.F32, al, None, al, other, 1, 4, 16, 64, 0.6, None) == L.ERR_UNSUPPORTED
    op.coef_dtype, op.kind = L.BF16, L.OP_SIGMA7
    assert f(L.BF16, al, None, al, other, 1, 4, 16, 64, 0.6, None) == L.ERR_UNSUPPORTED
    op.kind = L.OP_FACE7
    odd = C.c_void_p(al.value + 2)
    assert f(L.BF16, odd, None, al, other, 1, 4, 16, 64, 0.6, None) == L.ERR_BAD_ARG
    assert b"aligned" in lib.hfm_last_error()


def test_subcycle2d_validates_without_gpu(lib, pkg):
    """The fused 2D coarse cycle rejects first levels above 4096 cells, more than 8 levels, odd
    extents above the coarsest level, nu_pre < 1 and zero diagonal weights on the host."""
    L = pkg._lib
    w = (C.c_float * 72)(*([0, -1, 0, -1, 4, -1, 0, -1, 0] * 8))
    buf = (C.c_float * 16)()
    p = C.c_void_p(C.addressof(buf))
    f = lambda *a: lib.hfm_subcycle2d(L.F32, w, p, p, *a)
    assert f(1, 128, 64, 2, 0.8, 2, 2, 8, L.FLAG_PERIODIC, None) == L.ERR_BAD_ARG    # 8192 cells
    assert f(1, 64, 64, 9, 0.8, 2, 2, 8, L.FLAG_PERIODIC, None) == L.ERR_BAD_ARG     # 9 levels
    assert f(1, 64, 64, 8, 0.8, 2, 2, 8, L.FLAG_PERIODIC, None) == L.ERR_BAD_ARG     # 64 -> 0
    assert f(1, 12, 20, 4, 0.8, 2, 2, 8, L.FLAG_PERIODIC, None) == L.ERR_BAD_ARG     # 3 x 5 above 1 x 2
    assert b"odd" in lib.hfm_last_error()
    assert f(1, 64, 64, 3, 0.8, 0, 2, 8, L.FLAG_PERIODIC, None) == L.ERR_BAD_ARG     # nu_pre 0
    assert lib.hfm_subcycle2d(L.BF16, w, None, p, 1, 64, 64, 3, 0.8, 2, 2, 8, 0, None) == L.ERR_BAD_ARG
    w[9 + 4] = 0.0
    assert f(1, 64, 64, 3, 0.8, 2, 2, 8, L.FLAG_PERIODIC, None) == L.ERR_BAD_ARG
    assert b"diagonal" in lib.hfm_last_error()


def test_two_sweeps_flag_validates_without_gpu(lib, pkg):
    """HFM_FLAG_TWO_SWEEPS: a missing rhs, an rhs or a base that is the output and a coarse
    correction on odd extents are refused on the host."""
    L = pkg._lib
    w = (C.c_float * 9)(0, -1, 0, -1, 4, -1, 0, -1, 0)
    b1, b2 = (C.c_float * 64)(), (C.c_float * 64)()
    p, q = C.c_void_p(C.addressof(b1)), C.c_void_p(C.addressof(b2))
    f = lambda base, coarse, rhs, out: lib.hfm_jacobi2d(L.F32, w, base, coarse, 0.0, rhs, out, 1, 8,
                                                        8, 0.8, L.FLAG_TWO_SWEEPS, None)
    assert f(q, None, p, q) == L.ERR_BAD_ARG                                   # base == out
    assert lib.hfm_jacobi2d(L.F32, w, p, p, -1.0, p, q, 1, 7, 8, 0.8, L.FLAG_TWO_SWEEPS,
                            None) == L.ERR_BAD_ARG                            # odd Y, coarse
    assert f(None, None, None, q) == L.ERR_BAD_ARG
    assert f(None, None, q, q) == L.ERR_BAD_ARG
    assert b"two sweeps" in lib.hfm_last_error()


def test_pre2_restrict_validates_without_gpu(lib, pkg):
    """hfm_pre2_restrict2d refuses odd extents, NULL and aliased fields on the host."""
    L = pkg._lib
    w = (C.c_float * 9)(0, -1, 0, -1, 4, -1, 0, -1, 0)
    bufs = [(C.c_float * 64)() for _ in range(3)]
    f, p, c = (C.c_void_p(C.addressof(b)) for b in bufs)
    g = lambda *a: lib.hfm_pre2_restrict2d(L.F32, w, *a, 0.8, L.FLAG_PERIODIC, None)
    assert g(f, p, c, 1, 7, 8) == L.ERR_BAD_ARG
    assert b"even" in lib.hfm_last_error()
    assert g(f, f, c, 1, 8, 8) == L.ERR_BAD_ARG
    assert g(f, p, p, 1, 8, 8) == L.ERR_BAD_ARG
    assert g(None, p, c, 1, 8, 8) == L.ERR_BAD_ARG


def test_multigrid2d_plan_without_gpu(pkg):
    """Multigrid2D's plan on the host: the first level of at most 4096 cells starts the fused
    coarse cycle, whose weights are the per-level weights in order; an odd extent above the
    coarsest level or more than 8 fused levels keep one launch per level step."""
    KM = pkg.kolmogorov
    w = KM.laplace5(0.1)
    mg = KM.Multigrid2D((512, 512), w, device="cpu")
    assert mg.shapes[mg.l_sub] == (64, 64) and mg.L - mg.l_sub == 5 and mg.fused_coarse
    assert mg.fused_pairs
    ref = [v for l in range(mg.l_sub, mg.L) for v in mg.ws[l]]
    assert list(mg.ws_sub) == ref
    mg = KM.Multigrid2D((96, 80), w, device="cpu")
    assert mg.shapes[mg.l_sub] == (48, 40) and mg.shapes[-1] == (6, 5) and mg.fused_coarse
    mg = KM.Multigrid2D((100, 100), w, device="cpu")  # 25 x 25 above the coarsest level
    assert not mg.fused_coarse
    mg = KM.Multigrid2D((64, 64), w, min_edge=1, device="cpu")  # 64^2 .. 1^2: 7 levels
    assert mg.l_sub == 0 and mg.fused_coarse
    mg = KM.Multigrid2D((64, 64), w, device="cpu", fused_coarse=False, fused_pairs=False)
    assert not mg.fused_coarse and not mg.fused_pairs


def test_serve_config_and_validation_without_gpu(lib, pkg):
    """hfm_serve_*: the default configuration and the host-side checks that run before any
    device allocation."""
    L = pkg._lib
    c = L.HfmServeConfig()
    lib.hfm_serve_config_default(C.byref(c))
    assert list(c.edges[:c.n_edges]) == [32, 48, 64, 96, 128]
    assert c.slots == 64 and c.budget_bytes == 120e9 and c.cycles_per_tick == 4
    assert c.solver.accel == L.ACCEL_IR and c.solver.storage == L.BF16
    assert c.solver.tol == 1e-6 and c.solver.inner_tol == 1e-3 and c.solver.max_cycles == 600
    h = C.c_void_p()
    bad = L.HfmServeConfig.from_buffer_copy(c)
    bad.n_edges = 0
    assert lib.hfm_serve_create(C.byref(bad), C.byref(h)) == L.ERR_BAD_ARG
    bad = L.HfmServeConfig.from_buffer_copy(c)
    bad.edges[1] = 32
    assert lib.hfm_serve_create(C.byref(bad), C.byref(h)) == L.ERR_BAD_ARG
    assert b"repeated" in lib.hfm_last_error()
    bad = L.HfmServeConfig.from_buffer_copy(c)
    bad.solver.accel = L.ACCEL_CG
    assert lib.hfm_serve_create(C.byref(bad), C.byref(h)) == L.ERR_UNSUPPORTED
    bad = L.HfmServeConfig.from_buffer_copy(c)
    bad.budget_bytes = 1e6  # less than one 128^3 slot
    assert lib.hfm_serve_create(C.byref(bad), C.byref(h)) == L.ERR_OOM
    n = C.c_int()
    assert lib.hfm_serve_poll(None, None, 0, C.byref(n)) == L.ERR_BAD_ARG
    assert lib.hfm_serve_cancel(None, 0) == L.ERR_BAD_ARG
    assert lib.hfm_status_string(L.ERR_CANCELLED) == b"HFM_ERR_CANCELLED"
