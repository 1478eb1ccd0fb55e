"""hfm_norm2_f64_noalloc: the norm for callers that cannot allocate device memory.

Some callers have no device allocator to hand (a C or Fortran host code driving the solver)
or may not call cudaMalloc inside their time-step loop; this entry point keeps its partial
sums in the library's static device array instead of caller scratch.  The test calls it
through the C ABI twice in a row and compares each result with hfm_norm2_f64 (caller
scratch).  It lives in its own file, collected last, and needs no other test to run first.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _norm_both(hfm, x, B):
    import torch
    L = hfm._lib
    lib = L.lib()
    n = x.numel() // B
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    ref = torch.empty(B, dtype=torch.float64, device=x.device)
    scratch = torch.empty(lib.hfm_reduce_scratch_bytes(n, B), dtype=torch.uint8, device=x.device)
    L.call("hfm_norm2_f64", C.c_void_p(x.data_ptr()), n, B, C.c_void_p(ref.data_ptr()),
           C.c_void_p(scratch.data_ptr()), stream)
    got = torch.empty(B, dtype=torch.float64, device=x.device)
    L.call("hfm_norm2_f64_noalloc", C.c_void_p(x.data_ptr()), n, B, C.c_void_p(got.data_ptr()),
           stream)
    torch.cuda.synchronize()
    return got.cpu().numpy(), ref.cpu().numpy()


def test_noalloc_norm_matches_scratch_version_twice(hfm):
    import torch
    torch.manual_seed(0)
    # two calls in a row with different sizes: the second must not see the first's partials
    for B, n in ((7, 300001), (3, 4096)):
        x = torch.randn(B * n, device="cuda", dtype=torch.float32)
        got, ref = _norm_both(hfm, x, B)
        # same kernels, same summation order: the same bits
        np.testing.assert_array_equal(got, ref)
        np.testing.assert_allclose(got, np.linalg.norm(x.view(B, n).double().cpu().numpy(), axis=1),
                                   rtol=1e-12)


def test_noalloc_norm_rejects_oversize(hfm):
    import torch
    L = hfm._lib
    lib = L.lib()
    n, B = 1 << 22, 4096
    assert lib.hfm_reduce_scratch_bytes(n, B) > 512 * 1024
    out = torch.empty(B, dtype=torch.float64, device="cuda")
    x = torch.empty(16, device="cuda")  # never read: the size check comes first
    st = lib.hfm_norm2_f64_noalloc(C.c_void_p(x.data_ptr()), n, B, C.c_void_p(out.data_ptr()),
                                   C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == L.ERR_BAD_ARG
    assert b"static" in lib.hfm_last_error()
    # one grid row per instance: 65536 instances are rejected before any launch, even when
    # their partial sums would fit the array
    n, B = 8, 65536
    st = lib.hfm_norm2_f64_noalloc(C.c_void_p(x.data_ptr()), n, B, C.c_void_p(out.data_ptr()),
                                   C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == L.ERR_BAD_ARG
    assert b"65535" in lib.hfm_last_error()
    assert lib.hfm_reduce_scratch_bytes(n, B) == 0
