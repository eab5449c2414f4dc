"""Persistent scan: uint32 bit-exact vs the reference cpu_sum_scan semantics,
FP32 within 1e-5 relative (per element) of an FP64 prefix."""
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = pathlib.Path(__file__).resolve().parent / "golden"
REL_TOL_F32 = 1e-5


class _View:
    def __init__(self, ptr):
        self.ptr = ptr


def _scan(gsrb, ctx, a, f32=False, cfg=None, in_off=0, out_off=0, inplace=False):
    dt = np.float32 if f32 else np.uint32
    n = a.size
    din = ctx.array(n + in_off + 4, dt)
    buf = np.zeros(n + in_off + 4, dt)
    buf[in_off:in_off + n] = a
    din.upload(buf)
    if inplace:
        dout, out_off = din, in_off
    else:
        dout = ctx.array(n + out_off + 4, dt).zero()
    fn = gsrb.lib().gsrb_scan_f32 if f32 else gsrb.lib().gsrb_scan_u32
    import ctypes as C
    st = fn(ctx.h, din.ptr + 4 * in_off, dout.ptr + 4 * out_off, n, C.byref(cfg) if cfg is not None else None)
    gsrb.check(st, "scan")
    ctx.check_status("scan")
    return dout.download()[out_off:out_off + n]


def test_scan_u32_reference_golden(gsrb, ctx):
    z = np.load(GOLD / "scan_u32_golden.npz")
    for k in ("ones_1000", "u15_4099", "wrap_777", "single"):
        assert np.array_equal(_scan(gsrb, ctx, z[k + "_in"]), z[k + "_out"]), k


@pytest.mark.parametrize("n", [1, 3, 4, 5, 127, 128, 129, 4096, 24576 * 148 - 1, 32768 * 148, 32768 * 148 + 5,
                               2 * 32768 * 148 - 3, 10_000_019])
def test_scan_u32_sizes(gsrb, ctx, orc, n):
    a = gsrb.uniform_i32(n, n, 0, 15).astype(np.uint32)
    assert np.array_equal(_scan(gsrb, ctx, a), orc.scan_u32(a))


@pytest.mark.parametrize("in_off,out_off", [(1, 0), (0, 3), (2, 1)])
def test_scan_u32_unaligned(gsrb, ctx, orc, in_off, out_off):
    a = gsrb.uniform_i32(7, 777_777, 0, 15).astype(np.uint32)
    assert np.array_equal(_scan(gsrb, ctx, a, in_off=in_off, out_off=out_off), orc.scan_u32(a))


def test_scan_u32_inplace_and_wraparound(gsrb, ctx, orc):
    a = gsrb.uniform_i32(3, 2_000_003, 0, 2**31 - 1).astype(np.uint32) * np.uint32(3)
    assert np.array_equal(_scan(gsrb, ctx, a, inplace=True), orc.scan_u32(a))


@pytest.mark.parametrize("variant", [0, 2, 3, 4, 5, 6, 7, 8, 9, 11])
def test_scan_u32_barrier_variants(gsrb, ctx, orc, variant):
    a = gsrb.uniform_i32(11, 5_000_001, 0, 15).astype(np.uint32)
    c = gsrb.cfg(variant=variant, ctas_per_sm=1, threads=1024, cluster=2, tile=8192)
    assert np.array_equal(_scan(gsrb, ctx, a, cfg=c), orc.scan_u32(a))


@pytest.mark.parametrize("k,threads,tile", [(2, 512, 12288), (1, 256, 4096), (1, 1024, 16384), (2, 512, 65536),
                                            (1, 1024, 4), (4, 256, 1000)])
def test_scan_u32_shapes(gsrb, ctx, orc, k, threads, tile):
    a = gsrb.uniform_i32(k, 3_333_333, 0, 15).astype(np.uint32)
    c = gsrb.cfg(ctas_per_sm=k, threads=threads, cluster=2, tile=tile)
    assert np.array_equal(_scan(gsrb, ctx, a, cfg=c), orc.scan_u32(a))


@pytest.mark.parametrize("k,threads,tile,variant", [(1, 1024, 32768, 9), (2, 512, 16384, 9), (1, 128, 4096, 9),
                                                    (4, 256, 1000, 9), (1, 1024, 65536, 11), (2, 512, 8, 11)])
@pytest.mark.parametrize("n", [1, 4097, 3_333_333])
def test_scan_warp_specialised_shapes(gsrb, ctx, orc, k, threads, tile, variant, n):
    # FANOUT and HIER run the reader/writer warp-specialised kernel
    a = gsrb.uniform_i32(n + k, n, 0, 15).astype(np.uint32)
    c = gsrb.cfg(variant=variant, ctas_per_sm=k, threads=threads, tile=tile, wake_lines=4, fanin_groups=16)
    assert np.array_equal(_scan(gsrb, ctx, a, cfg=c), orc.scan_u32(a))
    f = gsrb.uniform_f32(n + 7, n)
    got = _scan(gsrb, ctx, f, f32=True, cfg=c)
    assert orc.max_rel_err(got[1:], orc.scan_f32_f64(f)[1:]) <= REL_TOL_F32


@pytest.mark.parametrize("n", [1, 5, 1000, 24576 * 148 + 3, 8_000_001])
def test_scan_f32_tolerance(gsrb, ctx, orc, n):
    a = gsrb.uniform_f32(n + 1, n)
    got = _scan(gsrb, ctx, a, f32=True)
    ref = orc.scan_f32_f64(a)
    assert orc.max_rel_err(got[1:], ref[1:]) <= REL_TOL_F32
    assert got[0] == 0.0


@pytest.mark.slow
def test_scan_full_size_2e28(gsrb, ctx, orc):
    # full size: 2^28 elements, u32 in [0,15] bit-exact, f32 in [0,1) 1e-5 relative
    n = 1 << 28
    a = gsrb.uniform_i32(0x5EED2022, n, 0, 15).astype(np.uint32)
    got = _scan(gsrb, ctx, a)
    assert np.array_equal(got, orc.scan_u32(a))
    del got
    f = gsrb.uniform_f32(0x5EED2022, n)
    got = _scan(gsrb, ctx, f, f32=True)
    ref = orc.scan_f32_f64(f)
    assert orc.max_rel_err(got[1:], ref[1:]) <= REL_TOL_F32


# ---- every protocol at sizes around the segment boundaries, and the
# warp-specialised kernel in place across chunk sizes (one vector to 64 Ki
# elements) with tails of 1-3 elements
@pytest.mark.parametrize("variant", [3, 4, 6, 8, 9, 11])
@pytest.mark.parametrize("n", [1, 7, 4096, 16384 * 148 * 3 + 5, 3_333_333])
def test_scan_variants_segment_edges(gsrb, ctx, orc, variant, n):
    a = gsrb.uniform_i32(n + variant, n, 0, 15).astype(np.uint32)
    c = gsrb.cfg(variant=variant, ctas_per_sm=1, threads=1024, wake_lines=4, fanin_groups=16, tile=16384)
    assert np.array_equal(_scan(gsrb, ctx, a, cfg=c), orc.scan_u32(a))
    f = gsrb.uniform_f32(n + 3, n)
    got = _scan(gsrb, ctx, f, f32=True, cfg=c)
    assert got[0] == 0.0
    assert orc.max_rel_err(got[1:], orc.scan_f32_f64(f)[1:]) <= REL_TOL_F32


@pytest.mark.parametrize("k,threads,tile", [(1, 1024, 4), (1, 1024, 1000), (1, 512, 8192), (2, 512, 16384),
                                            (2, 256, 24576), (1, 1024, 65536), (4, 256, 4096), (1, 128, 12)])
@pytest.mark.parametrize("inplace", [False, True])
def test_scan_ws_shapes(gsrb, ctx, orc, k, threads, tile, inplace):
    for n in (1_000_003, 148 * k * tile + 2):
        a = gsrb.uniform_i32(n + tile, n, 0, 2**31 - 1).astype(np.uint32) * np.uint32(7)  # wraps
        c = gsrb.cfg(variant=9, ctas_per_sm=k, threads=threads, tile=tile, wake_lines=4)
        assert np.array_equal(_scan(gsrb, ctx, a, cfg=c, inplace=inplace), orc.scan_u32(a)), n
