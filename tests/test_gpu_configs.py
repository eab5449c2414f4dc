"""The benchmark configurations themselves, as parity tests.

* C1: the sum of 2^24 int32 U[0,127] on exactly 148 x 2 CTAs x 256 threads,
  under each of the library's own barrier protocols, bit-exact, and the
  chained stream of such reductions that the bench times;
* C2: the barrier at full residency (148 x 8 x 256) -- 10,000-episode
  accounting and 10^5 message-passing episodes with no stale read -- and the
  priority semaphore at S in {1, 2, 10, 120}, one writer per 10 readers, 100
  increments per hold, exact counts;
* C4: RMAT-22 (a=0.57, b=c=0.19, edge factor 16) and the 2048 x 2048 grid:
  BFS levels and SSSP distances bit-exact against the oracle, pull PageRank
  within 1e-6 normalised L1 of FP64 (slow);
* C5: the 64-graph batch (RMAT scales 14-20), BFS and SSSP bit-exact per graph
  under the learned and the heuristic schedules (slow).
The 2^28 scans are in test_gpu_scan.py.
"""
import importlib.util
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = pathlib.Path(__file__).resolve().parents[1]
SEED = 0x5EED2022


def _policy():
    spec = importlib.util.spec_from_file_location("gsrb_policy", ROOT / "tpds22-artifact_b200" / "policy.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


# ------------------------------------------------------------------- C1
@pytest.fixture(scope="module")
def c1_input(gsrb):
    return gsrb.uniform_i32(SEED, 1 << 24, 0, 127)


@pytest.mark.parametrize("variant", [0, 3, 4, 8, 9, 11])
def test_c1_reduce_2e24_on_148x2x256(gsrb, ctx, orc, c1_input, variant):
    a = c1_input
    d = ctx.to_device(a)
    out = ctx.array(1, np.int64).zero()
    c = gsrb.cfg(variant=variant, ctas_per_sm=2, threads=256, cluster=2)
    gsrb.check(ctx.reduce_i32(d, a.size, out, c), "reduce")
    ctx.check_status("reduce")
    assert int(out.download()[0]) == orc.sum_i32(a)
    d.free()


@pytest.mark.parametrize("stages", [1, 2, 0])
def test_c1_chained_stream_of_2e24_reductions(gsrb, ctx, orc, stages):
    # the C1 workload as the bench times it: eight 2^24 inputs reduced in turn
    # by chained launches (cfg.overlap) on 148 x 2 x 256, replayed from a CUDA
    # graph twice; every sum bit-exact
    arrays = [gsrb.uniform_i32(SEED + i, 1 << 24, 0, 127) for i in range(8)]
    bufs = [ctx.to_device(a) for a in arrays]
    out = ctx.array(8, np.int64)
    c = gsrb.cfg(variant=gsrb.BAR_FANOUT, ctas_per_sm=2, threads=256, wake_lines=4, tile=stages, overlap=1)
    for i in range(8):  # warm the library's caches outside the capture
        gsrb.check(ctx.reduce_i32(bufs[i], 1 << 24, out.at(i), c), "reduce")
    cg = gsrb.CudaGraph(ctx)
    with cg:
        for i in range(8):
            gsrb.check(ctx.reduce_i32(bufs[i], 1 << 24, out.at(i), c), "reduce (capture)")
    try:
        for _ in range(2):
            out.upload(np.full(8, -1, np.int64))
            cg.launch()
            ctx.check_status("chained reduce")
            assert out.download().tolist() == [orc.sum_i32(a) for a in arrays]
    finally:
        cg.free()
    for b in bufs:
        b.free()


# ------------------------------------------------------------------- C2
@pytest.mark.parametrize("variant", [8, 9, 11, 3, 4])
def test_c2_barrier_full_residency_10k_episodes(gsrb, ctx, variant):
    c = gsrb.cfg(variant=variant, ctas_per_sm=8, threads=256, wake_lines=2)
    grid = 8 * ctx.num_sms
    sink = ctx.array(grid * 256, np.float32).zero()
    cnt = ctx.array(1, np.uint32).zero()
    gsrb.check(ctx.barrier_bench(c, 10_000, 0, sink, cnt), "barrier_bench")
    ctx.check_status("barrier_bench")
    assert int(cnt.download()[0]) == 10_000 * grid


@pytest.mark.parametrize("variant", [8, 9])
def test_c2_litmus_full_residency_1e5_episodes(gsrb, ctx, variant):
    c = gsrb.cfg(variant=variant, ctas_per_sm=8, threads=256, wake_lines=2)
    grid = 8 * ctx.num_sms
    buf = ctx.array(grid * 256, np.uint32).zero()
    stale = ctx.array(1, np.uint64).zero()
    gsrb.check(ctx.barrier_litmus(c, 100_000, buf, stale), "barrier_litmus")
    ctx.check_status("litmus")
    assert int(stale.download()[0]) == 0


@pytest.mark.parametrize("cap", [1, 2, 10, 120])
def test_c2_priority_semaphore_counts(gsrb, ctx, cap):
    k, iters, incs, every = 8, 2, 100, 11
    c = gsrb.cfg(ctas_per_sm=k, threads=256, timeout_ms=5000)
    cnt = ctx.array(8, np.uint32).zero()
    gsrb.check(ctx.semaphore_bench(c, gsrb.SEM_PRIORITY, cap, every, iters, incs, cnt), "semaphore_bench")
    W, R, inside, maxr, viol, acq, tmo, _ = cnt.download().tolist()
    grid = k * ctx.num_sms
    writers = len([b for b in range(grid) if b % every == 0])
    assert tmo == 0 and viol == 0 and inside == 0 and 1 <= maxr <= cap
    assert W == writers * iters * incs and R == (grid - writers) * iters * incs


# ------------------------------------------------------------------- C4
@pytest.fixture(scope="module")
def rmat22(gsrb):
    return gsrb.rmat(22, 16, a=0.57, b=0.19, c=0.19, seed=SEED, wlo=1, whi=255)


@pytest.fixture(scope="module")
def grid2048(gsrb):
    return gsrb.grid2d(2048, 2048, seed=SEED, wlo=1, whi=1000)


def _graph_case(gsrb, ctx, orc, g, pr=True):
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.int32)
    want = orc.bfs(g, 0)
    dg.set_policy(gsrb.mlp_init(3))  # any weights: the schedule changes, never the levels
    for mode in (gsrb.BFS_PUSH, gsrb.BFS_HEURISTIC, gsrb.BFS_LEARNED, gsrb.BFS_PUSH | gsrb.BFS_FLAG_LB):
        rc, _ = dg.bfs(0, out, mode)
        gsrb.check(rc, f"bfs mode {mode}")
        assert np.array_equal(out.download(), want), f"bfs mode {mode}"
    wd = orc.dijkstra(g, 0)
    for delta in (10000, 256):
        rc, _ = dg.sssp(0, out, delta)
        gsrb.check(rc, "sssp")
        assert np.array_equal(out.download(), wd), f"sssp delta {delta}"
    if pr:
        r = ctx.array(g.nnodes, np.float32)
        rc, _ = dg.pagerank(r, 0.85, 50)
        gsrb.check(rc, "pagerank")
        assert orc.normalized_l1(r.download(), orc.pagerank(g, 0.85, 50, threads=8)) <= 1e-6
    dg.free()


@pytest.mark.slow
def test_c4_rmat22(gsrb, ctx, orc, rmat22):
    _graph_case(gsrb, ctx, orc, rmat22)


@pytest.mark.slow
def test_c4_grid2048(gsrb, ctx, orc, grid2048):
    _graph_case(gsrb, ctx, orc, grid2048)


# ------------------------------------------------------------------- C5
@pytest.mark.slow
def test_c5_batch64_exact(gsrb, ctx, orc):
    rng = np.random.default_rng(SEED)
    scales = rng.integers(14, 21, 64)
    graphs = [gsrb.rmat(int(s), 16, seed=SEED + i, wlo=1, whi=255) for i, s in enumerate(scales)]
    dgs = [ctx.graph(g) for g in graphs]
    for dg in dgs:
        dg.set_policy(gsrb.mlp_init(5))
    outs = [ctx.array(g.nnodes, np.int32) for g in graphs]
    b = gsrb.Batch(ctx, dgs, gsrb.cfg(variant=gsrb.BAR_FANOUT, ctas_per_sm=2, threads=512, wake_lines=4))
    wants = [orc.bfs(g, 0) for g in graphs]
    for mode in (gsrb.BFS_LEARNED, gsrb.BFS_HEURISTIC):
        for o in outs:
            o.zero()
        gsrb.check(b.bfs([0] * 64, outs, mode), "batch bfs")
        gsrb.check(b.stats()[0], "batch stats")
        for o, w in zip(outs, wants):
            assert np.array_equal(o.download(), w)
    gsrb.check(b.sssp([0] * 64, outs, 256), "batch sssp")
    gsrb.check(b.stats()[0], "batch sssp stats")
    for g, o in zip(graphs, outs):
        assert np.array_equal(o.download(), orc.dijkstra(g, 0))
    b.free()
    for dg in dgs:
        dg.free()
