"""The allocation-free multi-dot entry point, through the C ABI.

``tt_vec_multidot_noalloc`` serves callers that cannot allocate device memory
(and so cannot create a ``tt_ctx``): an application that reserves the whole
GPU for its own pool, or a plugin host that only lends out buffers it owns.
Its partial sums live in a fixed array inside the library instead of the
context's scratch.  This test checks it against ``tt_vec_multidot`` on two
calls in a row (the shared array keeps the previous call's contents, which
must not leak into the next result) and that oversized requests are rejected.
The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _bind():
    import tt_b200
    f = tt_b200.lib.tt_vec_multidot_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p]
    g = tt_b200.lib.tt_vec_multidot
    g.restype = C.c_int
    g.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p]
    return tt_b200, f, g


def test_multidot_noalloc_matches_multidot_twice():
    import torch
    tt_b200, noalloc, multidot = _bind()
    ctx = tt_b200.Context(0)
    try:
        stream = C.c_void_p(ctx.stream())
        gen = torch.Generator(device="cuda").manual_seed(1234)
        for n, nvec in ((1_000_003, 7), (262_147, 16)):
            xs = [torch.randn(n, dtype=torch.float64, device="cuda", generator=gen) for _ in range(nvec)]
            y = torch.randn(n, dtype=torch.float64, device="cuda", generator=gen)
            ref = torch.empty(nvec, dtype=torch.float64, device="cuda")
            got = torch.full((nvec,), float("nan"), dtype=torch.float64, device="cuda")
            ptrs = (C.c_void_p * nvec)(*[x.data_ptr() for x in xs])
            torch.cuda.synchronize()
            assert multidot(ctx.h, n, nvec, ptrs, y.data_ptr(), ref.data_ptr()) == 0
            assert noalloc(stream, n, nvec, ptrs, y.data_ptr(), got.data_ptr()) == 0, \
                tt_b200.lib.tt_get_last_error()
            ctx.sync()
            r, g = ref.cpu().numpy(), got.cpu().numpy()
            scale = np.linalg.norm(torch.stack(xs).cpu().numpy(), axis=1) * float(torch.linalg.norm(y))
            assert np.all(np.abs(g - r) <= RTOL * scale), (g, r)
            exact = (torch.stack(xs) @ y).cpu().numpy()
            assert np.all(np.abs(g - exact) <= 1e-10 * scale)
    finally:
        ctx.close()


def test_multidot_noalloc_rejects_too_many_vectors():
    import torch
    tt_b200, noalloc, _ = _bind()
    x = torch.zeros(64, dtype=torch.float64, device="cuda")
    out = torch.zeros(17, dtype=torch.float64, device="cuda")
    ptrs = (C.c_void_p * 17)(*([x.data_ptr()] * 17))
    rc = noalloc(C.c_void_p(0), 64, 17, ptrs, x.data_ptr(), out.data_ptr())
    assert rc != 0
    assert b"1..16" in tt_b200.lib.tt_get_last_error()
