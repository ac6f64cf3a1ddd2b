"""ab2_dot_noalloc: the dot product for callers that cannot allocate.

Some hosts cannot call cudaMalloc when they need a reduction (their free HBM is
owned by another allocator, or the call site cannot afford the blocking and
device-wide synchronisation an allocation may bring).  ab2_dot_noalloc keeps
its scratch in a fixed array inside libab2 instead.  This file checks it
through the C ABI against ab2_dot (same reduction kernel, possibly another
summation tree) on two calls in a row, with two calls queued on one stream
before a single synchronisation, that many calls leave the device's free
memory unchanged, and that oversized inputs are refused.  It is collected last
so that a failure here never hides the other tests.
"""
import ctypes as C
import math

import numpy as np
import pytest

from alien_b200 import abi

pytestmark = pytest.mark.gpu

MAX_N = 4096 * 4096


def _noalloc(ctx, vx, vy, vout, n, slot=0):
    L = abi.lib()
    return L.ab2_dot_noalloc(C.c_void_p(vx.device_ptr), C.c_void_p(vy.device_ptr), n,
                             C.c_void_p(vout.device_ptr + 8 * slot), C.c_void_p(ctx.stream))


@pytest.mark.parametrize("n", [0, 1, 4095, 4097, 1_000_003, 7_077_888])
def test_dot_noalloc_matches_dot_twice(ctx, n):
    rng = np.random.default_rng(n)
    x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    vx, vy = ctx.vector(x), ctx.vector(y)
    ref = ctx.dot(vx, vy)
    scale = max(float(np.sum(np.abs(x * y))), 1e-300)
    out = ctx.vector(2)
    for call in range(2):  # the shared scratch keeps the previous call's contents
        out.upload(np.full(2, np.nan))
        assert _noalloc(ctx, vx, vy, out, n) == abi.AB2_OK
        got = out.download()[0]  # download synchronises the context's stream
        assert abs(got - ref) <= 1e-14 * scale, (call, got, ref)
        assert abs(got - math.fsum(x * y)) <= 1e-14 * scale


def test_dot_noalloc_rejects_oversize_and_bad_args(ctx):
    L = abi.lib()
    v = ctx.vector(4)
    p = C.c_void_p(v.device_ptr)
    assert L.ab2_dot_noalloc(p, p, MAX_N + 1, p, C.c_void_p(ctx.stream)) == abi.AB2_ERR_BAD_ARG
    assert L.ab2_dot_noalloc(p, p, -1, p, C.c_void_p(ctx.stream)) == abi.AB2_ERR_BAD_ARG
    assert L.ab2_dot_noalloc(p, p, 4, None, C.c_void_p(ctx.stream)) == abi.AB2_ERR_BAD_ARG


def test_dot_noalloc_two_calls_queued_on_one_stream(ctx):
    """Two calls with different inputs, one after the other on the same
    stream and only then one synchronisation: the second call's clearing of
    the shared counter and its partials are ordered after the first call's
    kernel, so both results are right."""
    rng = np.random.default_rng(11)
    n1, n2 = 5_000_001, 123_457
    x1, y1 = rng.uniform(-1, 1, n1), rng.uniform(-1, 1, n1)
    x2, y2 = rng.standard_normal(n2), rng.standard_normal(n2)
    v = [ctx.vector(a) for a in (x1, y1, x2, y2)]
    out = ctx.vector(np.full(2, np.nan))
    assert _noalloc(ctx, v[0], v[1], out, n1, slot=0) == abi.AB2_OK
    assert _noalloc(ctx, v[2], v[3], out, n2, slot=1) == abi.AB2_OK
    got = out.download()
    for g, x, y in ((got[0], x1, y1), (got[1], x2, y2)):
        scale = float(np.sum(np.abs(x * y)))
        assert abs(g - math.fsum(x * y)) <= 1e-14 * scale, (g, math.fsum(x * y))


def test_dot_noalloc_allocates_no_device_memory(ctx):
    """The device's free memory (cudaMemGetInfo, through torch) is the same
    before and after 200 calls, once the first call has done its set-up."""
    import torch

    n = 3_000_000
    rng = np.random.default_rng(5)
    x = rng.uniform(-1, 1, n)
    vx = ctx.vector(x)
    out = ctx.vector(1)
    torch.cuda.mem_get_info(0)  # torch's own context set-up happens here, not inside the measured span
    assert _noalloc(ctx, vx, vx, out, n) == abi.AB2_OK
    ctx.synchronize()
    free0, _ = torch.cuda.mem_get_info(0)
    for _ in range(200):
        assert _noalloc(ctx, vx, vx, out, n) == abi.AB2_OK
    ctx.synchronize()
    free1, _ = torch.cuda.mem_get_info(0)
    assert free1 == free0, (free0, free1)
    assert abs(out.download()[0] - math.fsum(x * x)) <= 1e-14 * math.fsum(x * x)
