"""Time one libhfm kernel on a synthetic batch with CUDA events (and serve as the ncu target).

    python ai-hfm-solver_b200/kernel_bench.py --kernel smooth --form sigma7 --n 64 --batch 64

Kernels: ``smooth`` (one weighted-Jacobi sweep), ``resid`` (A phi - b), ``restrict``
(fused residual + restriction), ``correct`` (fused prolongation + correction + sweep),
``apply27`` (27-point conv).  Prints one JSON line with the time per launch, the algorithmic
bytes per launch and the achieved GB/s.  Inputs are larger than L2 for the default sizes.
"""
import argparse
import ctypes as C
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

# algorithmic bytes per fine cell, float32
BYTES = {("smooth", "sigma7"): 24, ("smooth", "const7"): 12, ("smooth", "k27"): 12,
         ("resid", "sigma7"): 24, ("resid", "const7"): 12, ("resid", "k27"): 12,
         ("restrict", "sigma7"): 20.5, ("restrict", "const7"): 8.5,
         ("correct", "sigma7"): 24.5, ("correct", "const7"): 12.5, ("correct", "k27"): 12.5,
         ("apply27", "k27"): 8}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", default="smooth")
    ap.add_argument("--form", default="sigma7")
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--shape", default=None, help="Z,Y,X (overrides --n)")
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--dtype", default="f32", choices=["f32", "bf16", "f16"],
                    help="storage of fields and conductivities (smooth only)")
    a = ap.parse_args()
    import torch
    import __graft_entry__ as ge
    hfm = ge.load_package()
    ops, W = hfm.ops, hfm.weights
    Z, Y, X = (tuple(int(v) for v in a.shape.split(",")) if a.shape else (a.n, a.n, a.n))
    B = a.batch
    dev = torch.device("cuda")
    g = torch.Generator(device=dev).manual_seed(0)
    x = torch.randn((B, Z, Y, X), device=dev, generator=g)
    b = torch.randn((B, Z, Y, X), device=dev, generator=g)
    if a.form == "sigma7":
        s = torch.exp(torch.randn((3, B, Z, Y, X), device=dev, generator=g))
        op = ops.Sigma7(s[0], s[1], s[2])
    elif a.form == "const7":
        op = ops.Const7(50.0, 100.0, 200.0)
    else:
        op = ops.Stencil27(W.pressure27())
    out = torch.empty_like(x)
    wc = torch.randn((B, Z // 2, Y // 2, X // 2), device=dev, generator=g)
    st = op.struct()
    stream = ops._stream()
    L = hfm._lib
    P = lambda t: C.c_void_p(t.data_ptr() if t is not None else 0)

    tdt = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[a.dtype]
    if a.kernel == "smooth" and a.dtype != "f32":
        xt, bt, ot = x.to(tdt), b.to(tdt), out.to(tdt)
        keep = []
        if a.form == "sigma7":
            keep = [s[k].to(tdt).contiguous() for k in range(3)]
            for k in range(3):
                st.coef[k] = keep[k].data_ptr()
        st.coef_dtype = {"bf16": L.BF16, "f16": L.F16}[a.dtype]
        dcode = st.coef_dtype
        fn = lambda: L.call("hfm_op_jacobi_typed", C.byref(st), dcode, P(xt), P(bt), P(ot), B, Z, Y,
                            X, 2.0 / 3.0, 0, stream)
        BYTES[("smooth", a.form)] = BYTES[("smooth", a.form)] * (2 / 4)
    elif a.kernel == "smooth":
        fn = lambda: L.call("hfm_op_jacobi", C.byref(st), P(x), P(b), P(out), P(None), B, Z, Y, X,
                            2.0 / 3.0, 1, 0, stream)
    elif a.kernel == "resid":
        fn = lambda: L.call("hfm_op_residual", C.byref(st), P(x), P(b), P(out), B, Z, Y, X, 0, stream)
    elif a.kernel == "restrict":
        fn = lambda: L.call("hfm_residual_restrict", C.byref(st), P(x), P(b), P(None), P(wc),
                            B, Z, Y, X, 0, stream)
    elif a.kernel == "correct":
        fn = lambda: L.call("hfm_prolong_correct_smooth", C.byref(st), P(x), P(wc), P(b), P(out),
                            B, Z, Y, X, 2.0 / 3.0, 0, stream)
    elif a.kernel == "apply27":
        keep = W.pressure27().reshape(27).copy()
        fn = lambda: L.call("hfm_conv3d_k3", P(x), P(out), B, Z, Y, X,
                            keep.ctypes.data_as(C.c_void_p), stream)
    else:
        raise SystemExit("unknown kernel " + a.kernel)
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
    cells = B * Z * Y * X
    nbytes = BYTES.get((a.kernel, a.form), 0) * cells
    print(json.dumps({"kernel": a.kernel, "form": a.form, "shape": [B, Z, Y, X],
                      "ms_per_launch": ms, "bytes_per_launch": nbytes,
                      "gbs": nbytes / (ms / 1e3) / 1e9 if ms > 0 else None}))


if __name__ == "__main__":
    main()
