"""Batched traversals (one persistent launch, sub-grid barriers), CUDA-graph
replay, and the learned policy: results bit-exact per instance."""
import importlib.util
import pathlib
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = pathlib.Path(__file__).resolve().parents[1]


def _policy():
    spec = importlib.util.spec_from_file_location("gsrb_policy", ROOT / "tpds22-artifact_b200" / "policy.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def batch_graphs(gsrb):
    gs = [gsrb.rmat(s, 16, seed=100 + i) for i, s in enumerate([10, 11, 12, 13, 14, 12, 10, 13])]
    gs.append(gsrb.grid2d(40, 30, seed=5))
    gs.append(gsrb.csr_from_edges(500, np.arange(499), np.arange(1, 500)))
    return gs


@pytest.mark.parametrize("variant", [3, 4, 5, 8, 9, 11])
def test_batch_bfs_exact(gsrb, ctx, orc, batch_graphs, variant):
    dgs = [ctx.graph(g) for g in batch_graphs]
    outs = [ctx.array(g.nnodes, np.int32) for g in batch_graphs]
    c = gsrb.cfg(variant=variant, ctas_per_sm=2, threads=256)
    b = gsrb.Batch(ctx, dgs, c)
    f, n = b.layout()
    assert n.min() >= 1 and int(n.sum()) == 2 * ctx.num_sms and f[0] == 0
    srcs = [0] * len(dgs)
    gsrb.check(b.bfs(srcs, outs, gsrb.BFS_HEURISTIC), "batch_bfs")
    rc, st = b.stats()
    gsrb.check(rc, "batch_stats")
    ctx.check_status("batch")
    for g, o, s in zip(batch_graphs, outs, st):
        want = orc.bfs(g, 0)
        assert np.array_equal(o.download(), want)
        assert s.edges == orc.traversed_edges(g, want)


def test_batch_sssp_exact_and_graph_replay(gsrb, ctx, orc, batch_graphs):
    dgs = [ctx.graph(g) for g in batch_graphs]
    outs = [ctx.array(g.nnodes, np.int32) for g in batch_graphs]
    b = gsrb.Batch(ctx, dgs)
    srcs = [1] * len(dgs)
    gsrb.check(b.sssp(srcs, outs, 200), "batch_sssp")
    rc, _ = b.stats()
    gsrb.check(rc)
    for g, o in zip(batch_graphs, outs):
        assert np.array_equal(o.download(), orc.dijkstra(g, 1))
    # capture the batched launch in a CUDA graph and replay it twice
    for o in outs:
        o.zero()
    cg = gsrb.CudaGraph(ctx)
    with cg:
        gsrb.check(b.sssp(srcs, outs, 200))
    for _ in range(2):
        cg.launch()
        rc, _ = b.stats()
        gsrb.check(rc)
        for g, o in zip(batch_graphs, outs):
            assert np.array_equal(o.download(), orc.dijkstra(g, 1))
    cg.free()


def test_learned_policy_trains_and_stays_exact(gsrb, ctx, orc):
    pol = _policy()
    train = [gsrb.rmat(s, 16, seed=900 + s) for s in (12, 14, 15)] + [gsrb.grid2d(64, 64, seed=9)]
    X, Y, M = [], [], []
    for g in train:
        x, y, m, _ = pol.collect(ctx, ctx.graph(g), 0)
        X.append(x)
        Y.append(y)
        M.append(m)
    X, Y, M = np.concatenate(X), np.concatenate(Y), np.concatenate(M)
    params, hist = pol.train(ctx, X, Y, M, steps=800)
    assert hist[-1] < hist[0]
    evalg = [gsrb.rmat(13, 16, seed=77), gsrb.grid2d(50, 40, seed=2)]
    dgs = [ctx.graph(g) for g in evalg]
    for dg in dgs:
        dg.set_policy(params)
    outs = [ctx.array(g.nnodes, np.int32) for g in evalg]
    for dg, g, o in zip(dgs, evalg, outs):
        rc, st = dg.bfs(0, o, gsrb.BFS_LEARNED)
        gsrb.check(rc, "learned bfs")
        assert np.array_equal(o.download(), orc.bfs(g, 0))
        assert st.decisions >= 1
    b = gsrb.Batch(ctx, dgs)
    gsrb.check(b.bfs([0, 0], outs, gsrb.BFS_LEARNED))
    rc, _ = b.stats()
    gsrb.check(rc)
    for g, o in zip(evalg, outs):
        assert np.array_equal(o.download(), orc.bfs(g, 0))
