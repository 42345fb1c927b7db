"""rumb_butterfly_noalloc, the butterfly staged in the library's static device array, against
rumb_butterfly (context scratch) on the same slabs: two calls in a row per case, through the C ABI.
Collected last so that it runs both alone and after every other GPU test."""
import numpy as np
import pytest

from rumb import _lib

pytestmark = pytest.mark.gpu

COEFS = [(1.0, -1.0, 0.0, 1.0), (1.0, 1.0, 0.0, 1.0), (0.75, -0.5, 0.25, 1.5)]


@pytest.mark.parametrize("n", [2, 5, 9, 12, 16])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_noalloc_matches_butterfly(ctx, n, dtype):
    rng = np.random.default_rng(n)
    for k in COEFS:
        v = rng.standard_normal(n << (n - 1)).astype(dtype)
        ref = ctx.butterfly(n, v, *k)
        first = ctx.butterfly_noalloc(n, v, *k)
        second = ctx.butterfly_noalloc(n, v, *k)
        # same kernels and plan on the same slab: the tolerance is zero
        np.testing.assert_array_equal(first, ref)
        np.testing.assert_array_equal(second, ref)


def test_noalloc_size_limit(ctx):
    v = np.zeros(17 << 16)
    with pytest.raises(_lib.RumbError, match="static staging array holds 4194304"):
        ctx.butterfly_noalloc(17, v, 1.0, -1.0, 0.0, 1.0)
    # a rejected call leaves the entry point usable
    w = np.arange(16 << 15, dtype=np.float64)
    np.testing.assert_array_equal(ctx.butterfly_noalloc(16, w, 1.0, 1.0, 0.0, 1.0),
                                  ctx.butterfly(16, w, 1.0, 1.0, 0.0, 1.0))


def test_noalloc_allocates_no_device_memory():
    """The point of the entry point: after a warm-up call for each (n, dtype) used, further calls
    leave the device's free memory unchanged. The same check on rumb_butterfly, whose context
    scratch grows on first use, sees the free memory drop by the slab (4 MiB at n = 16 float64),
    which shows the check can fail."""
    c = _lib.Context(0)
    try:
        n = 16
        v = np.random.default_rng(3).standard_normal(n << (n - 1))
        ref = c.butterfly_noalloc(n, v, *COEFS[0])                # warm-up: symbol lookup, kernel loads
        c.sync()
        free0, _ = c.mem_info()
        for k in COEFS:
            c.butterfly_noalloc(n, v, *k)
        c.sync()
        free1, _ = c.mem_info()
        assert free1 == free0, (free0, free1)
        np.testing.assert_array_equal(c.butterfly_noalloc(n, v, *COEFS[0]), ref)
        c.butterfly(n, v, *COEFS[0])                               # first use of the context scratch
        c.sync()
        free2, _ = c.mem_info()
        assert free0 - free2 >= (n << (n - 1)) * 8, (free0, free2)
    finally:
        c.close()
