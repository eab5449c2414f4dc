"""The allocation-free reduce entry point (gsrb_reduce_i32_noalloc).

It exists for callers that must not allocate device memory (a host framework
that hands them a fixed memory budget, a plugin that may not grow the device
footprint or call cudaMalloc): its scratch is a fixed static device array.
Checked here through the C ABI against the context-based gsrb_reduce_i32 on
the same input, on two calls in a row (the static scratch keeps the previous
call's contents, so the second call must not see stale barrier state).

This file sorts last so that a run stopping at the first failure has already
run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(gsrb):
    gsrb.register("gsrb_reduce_i32_noalloc", C.c_int32, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p])
    return gsrb.lib().gsrb_reduce_i32_noalloc


def test_noalloc_matches_context_reduce_twice(gsrb, ctx):
    fn = _noalloc(gsrb)
    for call, (seed, n, lo, hi) in enumerate([(0x5EED2022, 1 << 24, 0, 127), (17, 3_000_001, -1000, 1000)]):
        a = gsrb.uniform_i32(seed, n, lo, hi)
        d = ctx.to_device(a)
        ref = ctx.array(1, np.int64).zero()
        gsrb.check(ctx.reduce_i32(d, n, ref), "reduce_i32")
        ctx.check_status("reduce_i32")
        got = ctx.array(1, np.int64).zero()
        ctx.sync()
        # default stream (NULL): synchronous entry point
        gsrb.check(fn(d.ptr, n, got.ptr, None), f"reduce_i32_noalloc call {call}")
        r, g = int(ref.download()[0]), int(got.download()[0])
        assert g == r, f"call {call}: {g} != {r}"
        assert r == int(a.astype(np.int64).sum())


def test_noalloc_rejects_oversized_input(gsrb, ctx):
    fn = _noalloc(gsrb)
    out = ctx.array(1, np.int64).zero()
    d = ctx.array(16, np.int32)
    assert fn(d.ptr, (1 << 32) + 1, out.ptr, None) == gsrb.ERR_ARG


@pytest.mark.parametrize("shift", [1, 3])
def test_noalloc_unaligned_and_small_inputs(gsrb, ctx, shift):
    # inputs that start 4 or 12 bytes past a 16-byte boundary (the kernel's
    # scalar head) and sizes at which most CTAs get empty slices
    fn = _noalloc(gsrb)
    sizes = [0, 1, 5, 2 * ctx.num_sms - 1, 1_000_003]
    for n in sizes:
        a = gsrb.uniform_i32(n + shift, n, -1000, 1000)
        buf = np.zeros(n + shift + 4, np.int32)
        buf[shift:shift + n] = a
        d = ctx.to_device(buf)
        got = ctx.array(1, np.int64).zero()
        ctx.sync()
        for call in range(2):
            gsrb.check(fn(d.ptr + 4 * shift, n, got.ptr, None), f"noalloc n={n} shift={shift} call {call}")
            assert int(got.download()[0]) == int(a.astype(np.int64).sum()), f"n={n} shift={shift} call {call}"
        d.free()
