"""Grid barrier parity on the GPU: episode accounting, message passing, bounded failure."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ALL = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12]


def _run_bench(gsrb, ctx, variant, k, cluster=2, episodes=2000, fma=0, threads=256, fanin=0):
    c = gsrb.cfg(variant=variant, ctas_per_sm=k, threads=threads, cluster=cluster, fanin_groups=fanin)
    grid = k * ctx.num_sms
    sink = ctx.array(grid * threads, np.float32).zero()
    cnt = ctx.array(1, np.uint32).zero()
    st = ctx.barrier_bench(c, episodes, fma, sink, cnt)
    return st, grid, cnt


@pytest.mark.parametrize("variant", ALL)
@pytest.mark.parametrize("k", [1, 2, 8])
def test_barrier_episode_count(gsrb, ctx, variant, k):
    st, grid, cnt = _run_bench(gsrb, ctx, variant, k)
    if st == gsrb.ERR_NOT_CORESIDENT:
        pytest.skip("configuration not co-resident on this device")
    gsrb.check(st, "barrier_bench")
    ctx.check_status("barrier_bench")
    assert int(cnt.download()[0]) == 2000 * grid


@pytest.mark.parametrize("cluster", [1, 2, 4, 8])
@pytest.mark.parametrize("fanin", [0, 8])
def test_cluster_sizes_and_fanin(gsrb, ctx, cluster, fanin):
    st, grid, cnt = _run_bench(gsrb, ctx, gsrb.BAR_CLUSTER, 2, cluster=cluster, fanin=fanin, episodes=1000)
    if st == gsrb.ERR_NOT_CORESIDENT:
        pytest.skip("not co-resident")
    gsrb.check(st)
    ctx.check_status()
    assert int(cnt.download()[0]) == 1000 * grid


@pytest.mark.parametrize("groups", [0, 8, 37, 148])
@pytest.mark.parametrize("wake", [1, 8])
@pytest.mark.parametrize("k", [1, 8])
def test_hier_groups_and_wake_lines(gsrb, ctx, groups, wake, k):
    c = gsrb.cfg(variant=gsrb.BAR_HIER, ctas_per_sm=k, threads=256, fanin_groups=groups, wake_lines=wake)
    grid = k * ctx.num_sms
    sink = ctx.array(grid * 256, np.float32).zero()
    cnt = ctx.array(1, np.uint32).zero()
    gsrb.check(ctx.barrier_bench(c, 1500, 4, sink, cnt))
    ctx.check_status()
    assert int(cnt.download()[0]) == 1500 * grid


@pytest.mark.parametrize("variant", ALL)
def test_barrier_message_passing_litmus(gsrb, ctx, variant):
    c = gsrb.cfg(variant=variant, ctas_per_sm=4, threads=128, cluster=4)
    grid = 4 * ctx.num_sms
    buf = ctx.array(grid * 128, np.uint32).zero()
    stale = ctx.array(1, np.uint64).zero()
    st = ctx.barrier_litmus(c, 3000, buf, stale)
    if st == gsrb.ERR_NOT_CORESIDENT:
        pytest.skip("not co-resident")
    gsrb.check(st)
    ctx.check_status()
    assert int(stale.download()[0]) == 0


def test_refuses_non_coresident_grid(gsrb, ctx):
    c = gsrb.cfg(variant=gsrb.BAR_FLAT, ctas_per_sm=64, threads=256)
    sink = ctx.array(64 * ctx.num_sms * 256, np.float32)
    cnt = ctx.array(1, np.uint32).zero()
    assert ctx.barrier_bench(c, 10, 0, sink, cnt) == gsrb.ERR_NOT_CORESIDENT


@pytest.mark.parametrize("variant", [0, 2, 3, 4, 5, 8, 9, 11, 12])
def test_short_grid_times_out_and_context_survives(gsrb, ctx, variant):
    # the expected arrival count is one participant higher than the launch:
    # every wait must run out (bounded) and report a timeout, not hang
    c = gsrb.cfg(variant=variant, ctas_per_sm=1, threads=64, cluster=2, timeout_ms=150)
    st = ctx.barrier_fault_short_grid(c)
    assert st == gsrb.ERR_TIMEOUT
    # the context is still usable afterwards
    st, grid, cnt = _run_bench(gsrb, ctx, gsrb.BAR_CLUSTER, 1, episodes=100)
    gsrb.check(st)
    ctx.check_status()
    assert int(cnt.download()[0]) == 100 * grid


@pytest.mark.parametrize("groups", [1, 16, 148])
@pytest.mark.parametrize("k", [1, 4])
def test_lockfree_flat_and_two_level(gsrb, ctx, groups, k):
    # fanin_groups = 1: one flat flag barrier (CTA 0 scans every flag);
    # > 1: per-group local barriers whose masters form the global one
    st, grid, cnt = _run_bench(gsrb, ctx, gsrb.BAR_LOCKFREE, k, fanin=groups, episodes=500)
    gsrb.check(st)
    ctx.check_status()
    assert int(cnt.download()[0]) == 500 * grid
