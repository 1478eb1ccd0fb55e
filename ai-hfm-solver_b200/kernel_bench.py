"""Time one libhfm kernel on a synthetic batch with CUDA events (and serve as the ncu target).

    python ai-hfm-solver_b200/kernel_bench.py --kernel smooth --form sigma7 --n 64 --batch 64
    python ai-hfm-solver_b200/kernel_bench.py --kernel smooth --form face7 --dtype bf16 --n 128

Kernels: ``smooth`` (one weighted-Jacobi sweep), ``resid`` (A phi - b), ``restrict`` (fused
residual + restriction), ``correct`` (fused prolongation + correction + sweep), ``apply27``
(27-point conv), ``transfer-r`` / ``transfer-p`` (standalone restriction / prolongation),
``smooth2`` (face7: coarse correction and two sweeps in one pass), ``served-shares``
(kernel-time shares of one pass over the served stream of --batch requests), ``mg-iter`` (bf16
refinement + PCG iterations on a handle of --batch slots of --n^3), ``kolmogorov-step``
(time steps of the 2D Kolmogorov flow at --n^2), ``subcycle2d`` (the fused 2D coarse cycle
from --n^2 down to 4^2, periodic 5-point operator, --batch instances), ``ns-step`` (time steps
of the obstacle flow at --shape, default 64,128,128: 24 boxes, 7-point
diffusion, F-cycle pressure solve to 1e-5; --reps steps in one timed region, the target of a
launch list).
Forms: ``sigma7`` (per-cell conductivities), ``face7`` (stored faces; 16-bit storage),
``const7``, ``k27``.  ``--dtype`` selects the storage of fields and coefficients (the typed
entry points for bf16 / f16).  Prints one JSON line with the time per launch, the
algorithmic bytes per launch (every array read once and every output written once, at its
actual size) and the achieved GB/s.  Inputs are larger than L2 for the default sizes.
"""
import argparse
import ctypes as C
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", default="smooth")
    ap.add_argument("--form", default="sigma7", choices=["sigma7", "face7", "const7", "k27"])
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--shape", default=None, help="Z,Y,X (overrides --n)")
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--dtype", default="f32", choices=["f32", "bf16", "f16"],
                    help="storage of fields and coefficients")
    ap.add_argument("--per-level", action="store_true",
                    help="kolmogorov-step: one launch per level step (no fused coarse cycle, no "
                         "fused pairs of sweeps)")
    a = ap.parse_args()
    import torch
    import __graft_entry__ as ge
    hfm = ge.load_package()
    ops, W, L = hfm.ops, hfm.weights, hfm._lib
    if a.kernel == "ns-step":
        return ns_step(hfm, torch, a)
    if a.kernel == "mg-iter":
        return mg_iter(hfm, torch, a)
    if a.kernel == "kolmogorov-step":
        return kolmogorov_step(hfm, torch, a)
    if a.kernel == "subcycle2d":
        return subcycle2d(hfm, torch, a)
    if a.kernel == "served-shares":
        return served_shares(hfm, torch, a)
    Z, Y, X = (tuple(int(v) for v in a.shape.split(",")) if a.shape else (a.n, a.n, a.n))
    B = a.batch
    n = Z * Y * X
    dev = torch.device("cuda")
    g = torch.Generator(device=dev).manual_seed(0)
    tdt = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[a.dtype]
    code = {"f32": L.F32, "bf16": L.BF16, "f16": L.F16}[a.dtype]
    E = torch.tensor([], dtype=tdt).element_size()
    x = torch.randn((B, Z, Y, X), device=dev, generator=g).to(tdt)
    b = torch.randn((B, Z, Y, X), device=dev, generator=g).to(tdt)
    out = torch.empty_like(x)
    wc = torch.randn((B, Z // 2, Y // 2, X // 2), device=dev, generator=g).to(tdt)
    P = lambda t: C.c_void_p(t.data_ptr() if t is not None else 0)
    stream = ops._stream()
    st = L.HfmOperator()
    st.scale = 1.0
    st.coef_dtype = code
    coef_bytes = 0  # coefficient bytes per launch
    keep = []
    if a.form in ("sigma7", "face7"):
        s = torch.exp(torch.randn((3, B, Z, Y, X), device=dev, generator=g))
        if a.form == "sigma7":
            keep = [s[k].to(tdt).contiguous() for k in range(3)]
            st.kind = L.OP_SIGMA7
            coef_bytes = 3 * B * n * E
        else:
            if a.dtype == "f32":
                raise SystemExit("face7 kernels are 16-bit")
            keep = [torch.empty((B, Z, Y, X + 8), dtype=tdt, device=dev),
                    torch.empty((B, Z, Y + 1, X), dtype=tdt, device=dev),
                    torch.empty((B, Z + 1, Y, X), dtype=tdt, device=dev)]
            L.call("hfm_sigma7_faces", code, P(s[0]), P(s[1]), P(s[2]), 1.0, 1.0, 1.0,
                   *(P(t) for t in keep), B, Z, Y, X, stream)
            st.kind = L.OP_FACE7
            coef_bytes = sum(t.numel() for t in keep) * E
        for k in range(3):
            st.c[k] = 1.0
            st.coef[k] = keep[k].data_ptr()
        del s
    elif a.form == "const7":
        st.kind = L.OP_CONST7
        st.k[0], st.k[1], st.k[2] = 50.0, 100.0, 200.0
    else:
        st.kind = L.OP_K27
        for i, v in enumerate(W.pressure27().reshape(27)):
            st.k[i] = float(v)
    field = B * n * E
    typed = a.dtype != "f32"
    if a.kernel == "smooth":
        fn = (lambda: L.call("hfm_op_jacobi_typed", C.byref(st), code, P(x), P(b), P(out), B, Z, Y, X,
                             2.0 / 3.0, 0, stream)) if typed else \
             (lambda: L.call("hfm_op_jacobi", C.byref(st), P(x), P(b), P(out), P(None), B, Z, Y, X,
                             2.0 / 3.0, 1, 0, stream))
        nbytes = 3 * field + coef_bytes
    elif a.kernel == "resid":
        fn = (lambda: L.call("hfm_op_residual_typed", C.byref(st), code, P(x), P(b), P(out), B, Z, Y,
                             X, 0, stream)) if typed else \
             (lambda: L.call("hfm_op_residual", C.byref(st), P(x), P(b), P(out), B, Z, Y, X, 0, stream))
        nbytes = 3 * field + coef_bytes
    elif a.kernel == "restrict":
        fn = (lambda: L.call("hfm_residual_restrict_typed", C.byref(st), code, P(x), P(b), P(None),
                             P(wc), B, Z, Y, X, 0, stream)) if typed else \
             (lambda: L.call("hfm_residual_restrict", C.byref(st), P(x), P(b), P(None), P(wc),
                             B, Z, Y, X, 0, stream))
        nbytes = 2 * field + field / 8 + coef_bytes
    elif a.kernel == "correct":
        fn = (lambda: L.call("hfm_prolong_correct_smooth_typed", C.byref(st), code, P(x), P(wc), P(b),
                             P(out), B, Z, Y, X, 2.0 / 3.0, 0, stream)) if typed else \
             (lambda: L.call("hfm_prolong_correct_smooth", C.byref(st), P(x), P(wc), P(b), P(out),
                             B, Z, Y, X, 2.0 / 3.0, 0, stream))
        nbytes = 3 * field + field / 8 + coef_bytes
    elif a.kernel == "smooth2":
        if a.form != "face7":
            raise SystemExit("smooth2 (two sweeps per pass) is a face7 kernel")
        fn = lambda: L.call("hfm_face7_smooth2_typed", C.byref(st), code, P(x), P(wc), P(b), P(out),
                            B, Z, Y, X, 2.0 / 3.0, stream)
        nbytes = 3 * field + field / 8 + coef_bytes
    elif a.kernel == "apply27":
        w27 = W.pressure27().reshape(27).copy()
        fn = lambda: L.call("hfm_conv3d_k3", P(x), P(out), B, Z, Y, X,
                            w27.ctypes.data_as(C.c_void_p), stream)
        nbytes = 2 * field
    elif a.kernel == "transfer-r":
        fn = lambda: L.call("hfm_restrict_avg", P(x), P(wc), B, Z, Y, X, stream)
        nbytes = field + field / 8
    elif a.kernel == "transfer-p":
        fn = lambda: L.call("hfm_prolong_nearest", P(wc), P(out), B, Z // 2, Y // 2, X // 2, stream)
        nbytes = field + field / 8
    else:
        raise SystemExit("unknown kernel " + a.kernel)
    if a.kernel in ("apply27", "transfer-r", "transfer-p") and typed:
        raise SystemExit("%s runs in float32 only" % a.kernel)
    for _ in range(a.warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    print(json.dumps({"kernel": a.kernel, "form": a.form, "dtype": a.dtype, "shape": [B, Z, Y, X],
                      "ms_per_launch": ms, "bytes_per_launch": nbytes,
                      "bytes_per_cell": nbytes / (B * n),
                      "gbs": nbytes / (ms / 1e3) / 1e9 if ms > 0 else None}))


def mg_iter(hfm, torch, a):
    """Float64 refinement around bf16 PCG-V(2,2) on a handle of --batch slots of --n^3 (the
    served 128^3 bucket by default: 64 slots), --reps iterations in one timed region after
    --warmup: the target of a launch list of the CG kernels (q = A p with p . q, k_cg_p,
    k_cg_xr, the float64 outer residual) next to the cycle's kernels."""
    M, L = hfm.multigrid, hfm._lib
    n, B = a.n, a.batch
    shape = (n, n, n)
    sig = torch.exp(torch.randn((3, B) + shape, device="cuda",
                                generator=torch.Generator(device="cuda").manual_seed(0)))
    f = torch.randn((B,) + shape, device="cuda", dtype=torch.float64,
                    generator=torch.Generator(device="cuda").manual_seed(1))
    cfg = M.SolverConfig(cycle="V", accel="ir", storage="bf16", tol=1e-300, max_cycles=100000,
                         inner_tol=1e-3)
    with M.Multigrid(shape, L.OP_SIGMA7, cfg, slots=B) as h:
        h.set_operator(hfm.ops.Sigma7(sig[0], sig[1], sig[2]))
        del sig
        for s in range(B):
            h.load_f64(s, f[s])
        h.run(a.warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed iterations
        h.run(a.reps)
        torch.cuda.nvtx.range_pop()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.reps
    print(json.dumps({"kernel": "mg-iter", "shape": [B, n, n, n], "ms_per_iteration": ms}))


def served_shares(hfm, torch, a):
    """Kernel-time shares of one pass over the served stream (--batch requests, the
    benchmark's stream and solver settings), from the CUDA activity trace of torch's
    profiler: every kernel of the pass, aggregated by name.  The pass runs once unprofiled
    first (graph capture, warm-up).  Times under a tracer are for shares only."""
    from torch.profiler import profile, ProfilerActivity
    sv, M = hfm.serving, hfm.multigrid
    reqs = sv.make_stream(count=a.batch, rate=2000.0, seed=0, device=torch.device("cuda"))
    cfg = M.SolverConfig(cycle="V", accel="ir", storage="bf16", tol=1e-6, max_cycles=600,
                         inner_tol=1e-3)
    server = sv.SolveServer(cfg=cfg, slots=64, budget_bytes=120e9, cycles_per_tick=4)
    try:
        server.serve(reqs, realtime=True)
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            server.serve(reqs, realtime=True)
            torch.cuda.synchronize()
    finally:
        server.close()
    tot, cnt = {}, {}
    for e in prof.events():
        if getattr(e.device_type, "name", "") != "CUDA" or e.name.startswith(("Memcpy", "Memset")):
            continue
        name = e.name.replace("(anonymous namespace)::", "").replace("hfm::", "")
        name = name.replace("void ", "").split("(")[0]
        t = getattr(e, "device_time_total", None)
        if t is None:
            t = getattr(e, "cuda_time_total", 0.0)
        tot[name] = tot.get(name, 0.0) + t
        cnt[name] = cnt.get(name, 0) + 1
    T = sum(tot.values())
    rows = sorted(tot.items(), key=lambda kv: -kv[1])
    print(json.dumps({"kernel": "served-shares", "requests": a.batch, "kernel_ms": T / 1e3,
                      "kernels": [{"name": k, "launches": cnt[k], "ms": v / 1e3,
                                   "share": v / T} for k, v in rows]}))


def kolmogorov_step(hfm, torch, a):
    """Time steps of the doubly periodic Kolmogorov flow at --n^2 (the 2D configuration:
    nu 1/40, sin(4y) forcing, dt 1e-3, three pressure V-cycles per step), --reps steps in
    one timed region (NVTX range "timed")."""
    kf = hfm.kolmogorov.KolmogorovFlow(n=a.n, dt=1e-3, cycles=3, seed=0)
    if a.per_level:
        kf.mg.fused_coarse = kf.mg.fused_pairs = False
    for _ in range(a.warmup):
        kf.step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    torch.cuda.nvtx.range_push("timed")
    for _ in range(a.reps):
        kf.step()
    torch.cuda.nvtx.range_pop()
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"kernel": "kolmogorov-step", "n": a.n, "fused_coarse": kf.mg.fused_coarse,
                      "fused_pairs": kf.mg.fused_pairs,
                      "ms_per_step": e0.elapsed_time(e1) / a.reps}))


def subcycle2d(hfm, torch, a):
    """hfm_subcycle2d alone: V(2,2) from --n^2 down to 4^2 with 32 coarsest sweeps, --batch
    instances (one block each), --reps launches in one timed region."""
    KM, L = hfm.kolmogorov, hfm._lib
    mg = KM.Multigrid2D((a.n, a.n), KM.laplace5(2 * 3.141592653589793 / a.n), slots=a.batch)
    assert mg.fused_coarse and mg.l_sub == 0
    g = torch.Generator(device="cuda").manual_seed(0)
    rhs = torch.randn((a.batch, a.n, a.n), device="cuda", generator=g)
    out = torch.empty_like(rhs)
    st = hfm.ops._stream()
    P = lambda t: C.c_void_p(t.data_ptr())
    go = lambda: L.call("hfm_subcycle2d", L.F32, mg.ws_sub, P(rhs), P(out), a.batch, a.n, a.n, mg.L,
                        mg.omega, mg.nu_pre, mg.nu_post, mg.coarse_sweeps, mg.flags, st)
    for _ in range(a.warmup):
        go()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        go()
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"kernel": "subcycle2d", "n": a.n, "batch": a.batch, "levels": mg.L,
                      "us_per_launch": 1e3 * e0.elapsed_time(e1) / a.reps}))


def ns_step(hfm, torch, a):
    """Time steps of the obstacle flow (the obstacle-flow configuration's settings)."""
    ns = hfm.ns
    shape = tuple(int(v) for v in a.shape.split(",")) if a.shape else (64, 128, 128)
    cfg = ns.NSConfig(dt=0.5, dx=1.0, Re=0.05, ub=1.0, diffusion="7", pressure="fcycle", p_tol=1e-5)
    sig = ns.obstacle_mask(shape, n_boxes=24, footprint=(4, 16), height=(8, 40), sigma=1e5, seed=0)
    st = ns.NSStepper(shape, cfg, sigma=sig)
    try:
        for _ in range(a.warmup):
            st.step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.reps):
            st.step()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.reps
        print(json.dumps({"kernel": "ns-step", "shape": list(shape), "ms_per_step": ms,
                          "pressure_cycles": st.p_cycles[-a.reps:]}))
    finally:
        st.close()


if __name__ == "__main__":
    main()
