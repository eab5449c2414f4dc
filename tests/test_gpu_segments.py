"""Batched reduce / scan segments (one persistent launch, a sub-grid barrier per
segment): bit-exact against the serial oracle per segment."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VARIANTS = [4, 8, 9]  # FLAT, FLIP, FANOUT


def _uneven_offsets(seed, k, lo=0, hi=1 << 18):
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi, k)
    lens[rng.integers(0, k, max(1, k // 8))] = 0  # some empty segments
    return np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)


def _reduce_segments(gsrb, ctx, a, off, cfg=None):
    d = ctx.to_device(a) if a.size else ctx.array(1, np.int32)
    out = ctx.array(len(off) - 1, np.int64).zero()
    gsrb.check(ctx.reduce_i32_segments(d, off, out, cfg), "reduce_i32_segments")
    ctx.check_status("reduce_i32_segments")
    return out.download()


def _scan_segments(gsrb, ctx, a, off, cfg=None):
    d = ctx.to_device(a) if a.size else ctx.array(1, np.uint32)
    out = ctx.array(max(a.size, 1), np.uint32).zero()
    gsrb.check(ctx.scan_u32_segments(d, out, off, cfg), "scan_u32_segments")
    ctx.check_status("scan_u32_segments")
    return out.download()[: a.size]


def _want_scan(orc, a, off):
    want = np.zeros(a.size, np.uint32)
    for i in range(len(off) - 1):
        s, e = int(off[i]), int(off[i + 1])
        if e > s:
            want[s:e] = orc.scan_u32(a[s:e])
    return want


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("k", [1, 7, 64, 127])
def test_reduce_segments_exact(gsrb, ctx, orc, variant, k):
    off = _uneven_offsets(k, k)
    a = gsrb.uniform_i32(0x5EED2022 + k, int(off[-1]), -1000, 1000)
    got = _reduce_segments(gsrb, ctx, a, off, gsrb.cfg(variant=variant, ctas_per_sm=2, threads=256))
    want = [orc.sum_i32(a[int(off[i]):int(off[i + 1])]) if off[i + 1] > off[i] else 0 for i in range(k)]
    assert got.tolist() == want


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("k", [1, 7, 64, 127])
def test_scan_segments_exact(gsrb, ctx, orc, variant, k):
    off = _uneven_offsets(100 + k, k)
    a = gsrb.uniform_i32(0x5EED2022 + k, int(off[-1]), 0, 15).astype(np.uint32)
    got = _scan_segments(gsrb, ctx, a, off, gsrb.cfg(variant=variant, ctas_per_sm=2, threads=256))
    assert np.array_equal(got, _want_scan(orc, a, off))


REL_TOL_F32 = 1e-5


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("k", [1, 9, 127])
def test_scan_f32_segments_within_tolerance(gsrb, ctx, orc, variant, k):
    # FP32 values U[0,1): every element within 1e-5 relative of the FP64 prefix
    # of its segment (the first element of a segment is exactly 0)
    off = _uneven_offsets(200 + k, k, hi=1 << 19)
    a = gsrb.uniform_f32(0x5EED2022 + k, int(off[-1]))
    d = ctx.to_device(a) if a.size else ctx.array(1, np.float32)
    out = ctx.array(max(a.size, 1), np.float32).zero()
    c = gsrb.cfg(variant=variant, ctas_per_sm=2, threads=256, tile=1 if k == 9 else 0)
    gsrb.check(ctx.scan_segments(d, out, off, c), "scan_f32_segments")
    ctx.check_status("scan_f32_segments")
    got = out.download()[: a.size]
    for i in range(k):
        s0, e0 = int(off[i]), int(off[i + 1])
        if e0 == s0:
            continue
        assert got[s0] == 0.0
        if e0 - s0 > 1:
            assert orc.max_rel_err(got[s0 + 1:e0], orc.scan_f32_f64(a[s0:e0])[1:]) <= REL_TOL_F32


@pytest.mark.parametrize("variant", VARIANTS)
@pytest.mark.parametrize("k", [1, 9, 127])
def test_scan_f32_segments_mixed_sign(gsrb, ctx, orc, variant, k):
    # FP32 values U[-1,1): prefixes cancel, so a relative bound means nothing
    # near zero.  Bound each element by the L1 mass it was summed from: the
    # FP32 tile scan and the FP32 result add at most a few ulps of the running
    # sum of |x| (chunk sums and carries are FP64), so 1e-5 of that mass holds
    off = _uneven_offsets(300 + k, k, hi=1 << 19)
    a = (gsrb.uniform_f32(0xC0FFEE + k, int(off[-1])) * np.float32(2.0) - np.float32(1.0)).astype(np.float32)
    d = ctx.to_device(a) if a.size else ctx.array(1, np.float32)
    out = ctx.array(max(a.size, 1), np.float32).zero()
    c = gsrb.cfg(variant=variant, ctas_per_sm=2, threads=256, tile=1 if k == 9 else 0)
    gsrb.check(ctx.scan_segments(d, out, off, c), "scan_f32_segments")
    ctx.check_status("scan_f32_segments")
    got = out.download()[: a.size].astype(np.float64)
    for i in range(k):
        s0, e0 = int(off[i]), int(off[i + 1])
        if e0 == s0:
            continue
        seg = a[s0:e0].astype(np.float64)
        want = np.concatenate([[0.0], np.cumsum(seg)[:-1]])
        mass = np.concatenate([[0.0], np.cumsum(np.abs(seg))[:-1]])
        err = np.abs(got[s0:e0] - want)
        assert got[s0] == 0.0
        assert np.all(err <= REL_TOL_F32 * mass + 1e-30), f"segment {i}: worst {float((err - REL_TOL_F32 * mass).max())}"


@pytest.mark.parametrize("variant", VARIANTS)
def test_scan_segments_many_rounds(gsrb, ctx, orc, variant):
    # one tile per CTA per round: tens of rounds per segment, so the double
    # buffered round sums are reused many times
    off = np.array([0, 1_000_003, 1_000_004, 1_700_000, 3_000_001], np.uint64)
    a = gsrb.uniform_i32(21, int(off[-1]), 0, 2**31 - 1).astype(np.uint32) * np.uint32(5)
    c = gsrb.cfg(variant=variant, ctas_per_sm=1, threads=128, tile=1)
    assert np.array_equal(_scan_segments(gsrb, ctx, a, off, c), _want_scan(orc, a, off))


@pytest.mark.parametrize("threads", [64, 512, 1024])
def test_segments_odd_offsets_and_tiny_segments(gsrb, ctx, orc, threads):
    # lengths 0..9 and a few large ones, so slices start at every alignment and
    # many segments have fewer elements than CTAs
    lens = np.array([0, 1, 2, 3, 5, 7, 9, 0, 0, 1, 100_003, 3, 1 << 20, 6, 8, 4, 2, 1], np.uint64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    cfg = gsrb.cfg(variant=9, ctas_per_sm=1, threads=threads)
    a = gsrb.uniform_i32(7, int(off[-1]), -(1 << 30), 1 << 30)
    got = _reduce_segments(gsrb, ctx, a, off, cfg)
    want = [orc.sum_i32(a[int(off[i]):int(off[i + 1])]) if off[i + 1] > off[i] else 0 for i in range(len(lens))]
    assert got.tolist() == want
    u = gsrb.uniform_i32(8, int(off[-1]), 0, 2**31 - 1).astype(np.uint32) * np.uint32(3)  # wraps
    assert np.array_equal(_scan_segments(gsrb, ctx, u, off, cfg), _want_scan(orc, u, off))


def test_segments_default_cfg_large_and_all_empty(gsrb, ctx, orc):
    # one 2^24 segment beside small ones, the default launch shape
    lens = np.array([1 << 24, 17, 0, 1 << 16], np.uint64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    a = gsrb.uniform_i32(0x5EED2022, int(off[-1]), 0, 127)
    got = _reduce_segments(gsrb, ctx, a, off)
    assert got.tolist() == [orc.sum_i32(a[int(off[i]):int(off[i + 1])]) if lens[i] else 0 for i in range(4)]
    u = gsrb.uniform_i32(5, int(off[-1]), 0, 15).astype(np.uint32)
    assert np.array_equal(_scan_segments(gsrb, ctx, u, off), _want_scan(orc, u, off))
    # every segment empty: sums are 0 and nothing is read
    off0 = np.zeros(9, np.uint64)
    assert _reduce_segments(gsrb, ctx, np.zeros(0, np.int32), off0).tolist() == [0] * 8


def test_segments_rejects_bad_arguments(gsrb, ctx):
    d = ctx.array(16, np.int32)
    out = ctx.array(200, np.int64)
    assert ctx.reduce_i32_segments(d, np.array([0, 8, 4], np.uint64), out) == gsrb.ERR_ARG  # decreasing
    assert ctx.reduce_i32_segments(d, np.arange(129, dtype=np.uint64), out) == gsrb.ERR_ARG  # k = 128
    c = gsrb.cfg(variant=9, ctas_per_sm=1, threads=256, grid_override=4)
    assert ctx.reduce_i32_segments(d, np.arange(6, dtype=np.uint64), out, c) == gsrb.ERR_ARG  # grid < k
    assert ctx.reduce_i32_segments(d, np.array([0, 16], np.uint64), out,
                                   gsrb.cfg(variant=6)) == gsrb.ERR_UNSUPPORTED  # grid.sync is whole-grid
    u = ctx.array(16, np.uint32)
    assert ctx.scan_u32_segments(u, u, np.array([0, 16], np.uint64)) == gsrb.ERR_ARG  # in place


def test_segments_graph_replay(gsrb, ctx, orc):
    off = _uneven_offsets(3, 40)
    a = gsrb.uniform_i32(11, int(off[-1]), 0, 127)
    d = ctx.to_device(a)
    out = ctx.array(40, np.int64).zero()
    want = [orc.sum_i32(a[int(off[i]):int(off[i + 1])]) if off[i + 1] > off[i] else 0 for i in range(40)]
    cg = gsrb.CudaGraph(ctx)
    with cg:
        gsrb.check(ctx.reduce_i32_segments(d, off, out))
    for _ in range(3):
        out.zero()
        cg.launch()
        ctx.check_status("replay")
        assert out.download().tolist() == want
    cg.free()


# ---- register-resident rounds (cfg.form = FORM_REG, fan-out sub-grid barrier):
# groups of each CTA take the rounds in turn and keep their chunk in registers
# from its sum to its rescan.  Shapes: (CTAs/SM, threads, groups); the chunk is
# threads x 4 x (16 vectors a lane when CTAs/SM x threads <= 512, else 8) / groups.
REG_SHAPES = [(1, 512, 2), (1, 512, 4), (2, 256, 2), (4, 128, 2), (1, 1024, 2), (1, 1024, 4), (1, 768, 3),
              (1, 64, 2), (2, 512, 4)]


def _reg_cfg(gsrb, k, threads, groups):
    per = threads * (16 if threads * k <= 512 else 8) * 4
    return gsrb.cfg(variant=9, ctas_per_sm=k, threads=threads, form=gsrb.FORM_REG, tile=per // groups, wake_lines=4)


class _At:
    """A device address inside an array, with its element type."""

    def __init__(self, arr, elems):
        self.ptr = arr.ptr + 4 * elems
        self.dtype = arr.dtype


@pytest.mark.parametrize("k_sm,threads,groups", REG_SHAPES)
@pytest.mark.parametrize("k", [1, 7, 64, 127])
def test_scan_segments_reg_exact(gsrb, ctx, orc, k_sm, threads, groups, k):
    off = _uneven_offsets(500 + k, k)
    a = gsrb.uniform_i32(0x5EED2022 + k, int(off[-1]), 0, 2**31 - 1).astype(np.uint32) * np.uint32(3)  # wraps
    got = _scan_segments(gsrb, ctx, a, off, _reg_cfg(gsrb, k_sm, threads, groups))
    assert np.array_equal(got, _want_scan(orc, a, off))


@pytest.mark.parametrize("in_off,out_off", [(0, 0), (1, 1), (3, 3), (1, 0), (0, 2), (2, 3)])
def test_scan_segments_reg_alignment_and_tiny_segments(gsrb, ctx, orc, in_off, out_off):
    # segments start at every alignment; input and output at the same or a
    # different 16-byte phase (128-bit stores only when they match)
    lens = np.array([0, 1, 2, 3, 5, 7, 9, 0, 1, 100_003, 3, 1 << 20, 6, 8, 4, 2, 1, 777_777], np.uint64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    n = int(off[-1])
    u = gsrb.uniform_i32(9, n, 0, 2**31 - 1).astype(np.uint32) * np.uint32(7)
    buf = np.zeros(n + 8, np.uint32)
    buf[in_off:in_off + n] = u
    d = ctx.to_device(buf)
    out = ctx.array(n + 8, np.uint32)
    for shape in ((1, 512, 2), (2, 256, 4), (1, 1024, 2)):
        out.zero()
        c = _reg_cfg(gsrb, *shape)
        gsrb.check(ctx.scan_u32_segments(_At(d, in_off), _At(out, out_off), off, c), "scan_u32_segments")
        ctx.check_status("scan_u32_segments")
        full = out.download()
        assert np.array_equal(full[out_off:out_off + n], _want_scan(orc, u, off)), shape
        # nothing outside the output range is written
        assert not full[:out_off].any() and not full[out_off + n:].any()


@pytest.mark.parametrize("k", [1, 9, 127])
def test_scan_f32_segments_reg_tolerance_and_mixed_sign(gsrb, ctx, orc, k):
    off = _uneven_offsets(600 + k, k, hi=1 << 19)
    c = _reg_cfg(gsrb, 1, 512, 2)
    for mixed in (False, True):
        a = gsrb.uniform_f32(0xC0FFEE + k, int(off[-1]))
        if mixed:
            a = (a * np.float32(2.0) - np.float32(1.0)).astype(np.float32)
        d = ctx.to_device(a) if a.size else ctx.array(1, np.float32)
        out = ctx.array(max(a.size, 1), np.float32).zero()
        gsrb.check(ctx.scan_segments(d, out, off, c), "scan_f32_segments")
        ctx.check_status("scan_f32_segments")
        got = out.download()[: a.size].astype(np.float64)
        for i in range(k):
            s0, e0 = int(off[i]), int(off[i + 1])
            if e0 == s0:
                continue
            seg = a[s0:e0].astype(np.float64)
            want = np.concatenate([[0.0], np.cumsum(seg)[:-1]])
            mass = np.concatenate([[0.0], np.cumsum(np.abs(seg))[:-1]])
            assert got[s0] == 0.0
            assert np.all(np.abs(got[s0:e0] - want) <= REL_TOL_F32 * mass + 1e-30), (i, mixed)


def test_scan_segments_reg_many_rounds_and_replay(gsrb, ctx, orc):
    # small chunks: tens of rounds per segment, the round sums' buffers reused
    # many times; then the same call replayed from a CUDA graph
    off = np.array([0, 1_000_003, 1_000_004, 1_700_000, 3_000_001], np.uint64)
    a = gsrb.uniform_i32(21, int(off[-1]), 0, 2**31 - 1).astype(np.uint32) * np.uint32(5)
    want = _want_scan(orc, a, off)
    c = _reg_cfg(gsrb, 1, 128, 4)
    assert np.array_equal(_scan_segments(gsrb, ctx, a, off, c), want)
    d = ctx.to_device(a)
    out = ctx.array(a.size, np.uint32)
    gsrb.check(ctx.scan_u32_segments(d, out, off, c))
    cg = gsrb.CudaGraph(ctx)
    with cg:
        gsrb.check(ctx.scan_u32_segments(d, out, off, c))
    for _ in range(2):
        out.zero()
        cg.launch()
        ctx.check_status("replay")
        assert np.array_equal(out.download(), want)
    cg.free()


def test_scan_segments_reg_bad_cfg(gsrb, ctx):
    u = ctx.array(64, np.uint32)
    o = ctx.array(64, np.uint32)
    off = np.array([0, 64], np.uint64)
    assert ctx.scan_u32_segments(u, o, off, gsrb.cfg(variant=8, ctas_per_sm=1, threads=512,
                                                     form=gsrb.FORM_REG)) == gsrb.ERR_UNSUPPORTED
    for tile in (1000, 512 * 64 * 2, 512 * 64 // 8):  # not threads x 64 / (2..4)
        c = gsrb.cfg(variant=9, ctas_per_sm=1, threads=512, form=gsrb.FORM_REG, tile=tile)
        assert ctx.scan_u32_segments(u, o, off, c) == gsrb.ERR_ARG
