"""The context's cache of large device blocks (tt_ctx_set_block_cache).

Allocations of 32 MB or more are rounded up to a size class (2^k + j 2^(k-2))
and kept by the context when freed, so the next allocation of the same class
on the context's stream takes the same block without a call into the device
pool.  Checked here: a freed block is reused by a request of the same class
and not by one of another class; data written through a reused block is the
data read back; the cap is honoured; turning the cache off returns the blocks.
The contraction tests and the DMRG tests run with the cache on (the default).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MB = 1 << 20


def _alloc(lib, ctx, nbytes):
    p = C.c_void_p()
    assert lib.tt_device_alloc(ctx.h, nbytes, C.byref(p)) == 0
    return p.value


def _free(lib, ctx, p):
    assert lib.tt_device_free(ctx.h, C.c_void_p(p)) == 0


def test_block_cache_reuses_blocks_by_size_class():
    import tt_b200
    lib = tt_b200.lib
    ctx = tt_b200.Context(0)
    try:
        s0 = ctx.alloc_stats()
        a = _alloc(lib, ctx, 100 * MB)          # class 112 MB (64 + 3 * 16)
        _free(lib, ctx, a)
        assert ctx.alloc_stats()["cached_bytes"] == s0["cached_bytes"] + 112 * MB
        b = _alloc(lib, ctx, 97 * MB)           # same class: the cached block
        assert b == a
        assert ctx.alloc_stats()["cache_hits"] == s0["cache_hits"] + 1
        c = _alloc(lib, ctx, 120 * MB)          # class 128 MB: a new block
        assert c != a
        assert ctx.alloc_stats()["cache_hits"] == s0["cache_hits"] + 1
        # data through a reused block: fill on the host, copy in and back
        host = np.arange(97 * MB // 8, dtype=np.float64)
        out = np.empty_like(host)
        assert lib.tt_memcpy_h2d(ctx.h, C.c_void_p(b), host.ctypes.data_as(C.c_void_p), host.nbytes) == 0
        assert lib.tt_memcpy_d2h(ctx.h, out.ctypes.data_as(C.c_void_p), C.c_void_p(b), out.nbytes) == 0
        ctx.sync()
        assert np.array_equal(out, host)
        _free(lib, ctx, b)
        _free(lib, ctx, c)
        assert ctx.alloc_stats()["cached_bytes"] == s0["cached_bytes"] + 240 * MB
        # a smaller class takes the smallest cached block up to 1.5x its class
        f = _alloc(lib, ctx, 90 * MB)           # class 96 MB: the 112 MB block
        assert f == a
        _free(lib, ctx, f)
        g = _alloc(lib, ctx, 40 * MB)           # class 40 MB: nothing cached fits
        assert g not in (a, c)
        # at the cap, the block freed longest ago goes back to the pool
        ctx.set_block_cache(240 * MB)
        _free(lib, ctx, g)                      # evicts the 128 MB block (the oldest)
        assert ctx.alloc_stats()["cached_bytes"] == 152 * MB
        h = _alloc(lib, ctx, 120 * MB)          # class 128: the 112 and 40 MB blocks do not fit
        assert ctx.alloc_stats()["cached_bytes"] == 152 * MB
        _free(lib, ctx, h)                      # 152 + 128 > 240: evicts the 112 MB block
        assert ctx.alloc_stats()["cached_bytes"] == 168 * MB
        # a cap below what is cached releases everything; a freed block above
        # the cap goes back to the pool
        ctx.set_block_cache(64 * MB)
        assert ctx.alloc_stats()["cached_bytes"] == 0
        d = _alloc(lib, ctx, 100 * MB)
        _free(lib, ctx, d)
        assert ctx.alloc_stats()["cached_bytes"] == 0
        small = _alloc(lib, ctx, 36 * MB)       # class 40 MB (32 + 8), within the cap
        _free(lib, ctx, small)
        assert ctx.alloc_stats()["cached_bytes"] == 40 * MB
        ctx.set_block_cache(0)
        assert ctx.alloc_stats()["cached_bytes"] == 0
        # with the cache off, allocations are exact and nothing is kept
        e = _alloc(lib, ctx, 100 * MB)
        _free(lib, ctx, e)
        assert ctx.alloc_stats()["cached_bytes"] == 0
        ctx.sync()
    finally:
        ctx.close()
