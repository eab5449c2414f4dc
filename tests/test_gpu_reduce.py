"""Persistent reduce: bit-exact against the serial int64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VARIANTS = [0, 2, 3, 4, 5, 6, 7, 8, 9, 11]


def _reduce(gsrb, ctx, a, cfg=None, offset=0):
    d = ctx.array(a.size + offset, np.int32)
    if a.size:
        buf = np.zeros(a.size + offset, np.int32)
        buf[offset:] = a
        d.upload(buf)
    out = ctx.array(1, np.int64).zero()
    import ctypes
    view = type("V", (), {})()
    view.ptr = d.ptr + 4 * offset
    gsrb.check(ctx.reduce_i32(view, a.size, out, cfg), "reduce")
    ctx.check_status("reduce")
    return int(out.download()[0])


@pytest.mark.parametrize("variant", VARIANTS)
def test_reduce_seeded_uniform(gsrb, ctx, orc, variant):
    a = gsrb.uniform_i32(0x5EED2022, 1_000_003, 0, 127)
    c = gsrb.cfg(variant=variant, ctas_per_sm=2, threads=256, cluster=2)
    assert _reduce(gsrb, ctx, a, c) == orc.sum_i32(a)


def test_reduce_full_config(gsrb, ctx, orc):
    # 2^24 int32 U[0,127], the library's default grid (one 1024-thread CTA per SM)
    a = gsrb.uniform_i32(0x5EED2022, 1 << 24, 0, 127)
    assert _reduce(gsrb, ctx, a) == orc.sum_i32(a)


@pytest.mark.parametrize("n", [0, 1, 3, 4, 5, 255, 256, 257, 4096 + 7, 303_104])
@pytest.mark.parametrize("offset", [0, 1, 3])
def test_reduce_edge_sizes_and_alignment(gsrb, ctx, orc, n, offset):
    a = gsrb.uniform_i32(n + 17, n, -1000, 1000)
    assert _reduce(gsrb, ctx, a, offset=offset) == orc.sum_i32(a)


def test_reduce_all_ones_reference_golden(gsrb, ctx):
    # Reduce/test_reduce.cu:14-17
    for n in (1, 1000, 303_104, 1 << 22):
        assert _reduce(gsrb, ctx, np.ones(n, np.int32)) == n


def test_reduce_int64_no_overflow(gsrb, ctx, orc):
    a = np.full(1 << 21, 2**31 - 1, dtype=np.int32)
    assert _reduce(gsrb, ctx, a) == (2**31 - 1) * (1 << 21)
    b = np.full(1 << 20, -2**31, dtype=np.int32)
    assert _reduce(gsrb, ctx, b) == -(2**31) * (1 << 20)


@pytest.mark.parametrize("k,threads,stages", [(1, 1024, 0), (4, 128, 0), (4, 256, 0), (1, 512, 1), (1, 1024, 7),
                                              (2, 256, 2), (1, 64, 6)])
def test_reduce_other_shapes(gsrb, ctx, orc, k, threads, stages):
    a = gsrb.uniform_i32(99, 7_777_777, 0, 127)
    c = gsrb.cfg(ctas_per_sm=k, threads=threads, cluster=2, tile=stages)
    assert _reduce(gsrb, ctx, a, c) == orc.sum_i32(a)


# protocols of chained launches (cfg.overlap = 1): (variant, cluster, extra cfg)
CHAIN = [(9, 1, dict(wake_lines=4)), (8, 1, dict(fanin_groups=1)), (11, 1, dict(fanin_groups=16, wake_lines=4)),
         (0, 2, {}), (3, 1, {}), (4, 1, {})]


@pytest.mark.parametrize("variant,cluster,extra", CHAIN)
@pytest.mark.parametrize("graph", [False, True])
def test_reduce_chained_launches(gsrb, ctx, orc, variant, cluster, extra, graph):
    # A chain of reductions over distinct inputs of uneven sizes, each launch
    # allowed to start (and read its input) while the previous one finishes;
    # they share the barrier state and the partials, which a launch touches only
    # after the previous one has completed.  Every result bit-exact, three times
    # over (a chain also follows the previous chain's last launch).
    sizes = [1 << 22, 3_000_001, 17, 0, 1 << 20, 5_555_555, 1 << 22, 1]
    arrays = [gsrb.uniform_i32(1000 + i, n, -1000, 1000) for i, n in enumerate(sizes)]
    bufs = [ctx.to_device(a) if a.size else ctx.array(1, np.int32).zero() for a in arrays]
    out = ctx.array(len(sizes), np.int64)
    c = gsrb.cfg(variant=variant, ctas_per_sm=2, threads=256, cluster=cluster, overlap=1, **extra)
    want = [orc.sum_i32(a) for a in arrays]

    def chain():
        for i, n in enumerate(sizes):
            gsrb.check(ctx.reduce_i32(bufs[i], n, out.at(i), c), f"chained reduce {i}")

    cg = None
    if graph:
        chain()  # warm the library's caches outside the capture
        cg = gsrb.CudaGraph(ctx)
        with cg:
            chain()
    try:
        for rep in range(3):
            out.upload(np.full(len(sizes), -1, np.int64))
            if cg:
                cg.launch()
            else:
                chain()
            ctx.check_status("chained reduce")
            assert out.download().tolist() == want, f"rep {rep}"
    finally:
        if cg:
            cg.free()
    for b in bufs:
        b.free()


def test_reduce_overlap_refused_for_cooperative_launch(gsrb, ctx):
    # a chained launch is a plain launch; grid.sync's cooperative launch refuses it
    a = ctx.to_device(np.ones(1000, np.int32))
    out = ctx.array(1, np.int64)
    c = gsrb.cfg(variant=gsrb.BAR_CCG, ctas_per_sm=2, threads=256, overlap=1)
    assert ctx.reduce_i32(a, 1000, out, c) == gsrb.ERR_UNSUPPORTED
    a.free()
