"""Persistent BFS / SSSP / PageRank vs the CPU oracle (levels and distances
bit-exact; PageRank within 1e-6 normalized L1 of FP64)."""
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLD = pathlib.Path(__file__).resolve().parent / "golden"
PR_L1_TOL = 1e-6


def _graphs(gsrb):
    return {
        "tiny": gsrb.Graph.read_gr(GOLD / "tiny.gr"),
        "rmat12": gsrb.rmat(12, 16, seed=7),
        "rmat16": gsrb.rmat(16, 16, seed=11),
        "grid64": gsrb.grid2d(64, 48, seed=3),
        "path": gsrb.csr_from_edges(3000, np.arange(2999), np.arange(1, 3000)),
        "isolated": gsrb.csr_from_edges(100, [0, 1, 50], [1, 2, 51]),
    }


@pytest.fixture(scope="module")
def graphs(gsrb):
    return _graphs(gsrb)


@pytest.mark.parametrize("name", ["tiny", "rmat12", "rmat16", "grid64", "path", "isolated"])
@pytest.mark.parametrize("mode", [0, 1, 3, 4])
def test_bfs_levels_exact(gsrb, ctx, orc, graphs, name, mode):
    g = graphs[name]
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.int32)
    rc, st = dg.bfs(0, out, mode)
    gsrb.check(rc, "bfs")
    ctx.check_status("bfs")
    want = orc.bfs(g, 0)
    assert np.array_equal(out.download(), want)
    assert st.edges == orc.traversed_edges(g, want)


@pytest.mark.parametrize("variant", [0, 2, 3, 4, 5, 6, 7, 8, 9, 11])
def test_bfs_barrier_variants(gsrb, ctx, orc, graphs, variant):
    g = graphs["rmat16"]
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.int32)
    c = gsrb.cfg(variant=variant, ctas_per_sm=2, threads=256, cluster=2)
    rc, st = dg.bfs(5, out, gsrb.BFS_HEURISTIC, c)
    gsrb.check(rc)
    assert np.array_equal(out.download(), orc.bfs(g, 5))


@pytest.mark.parametrize("name,delta", [("tiny", 5), ("rmat12", 64), ("rmat16", 300), ("grid64", 2000),
                                        ("path", 100), ("isolated", 10), ("rmat16", 1 << 30)])
def test_sssp_distances_exact(gsrb, ctx, orc, graphs, name, delta):
    g = graphs[name]
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.int32)
    rc, st = dg.sssp(0, out, delta)
    gsrb.check(rc, "sssp")
    ctx.check_status("sssp")
    assert np.array_equal(out.download(), orc.dijkstra(g, 0))


@pytest.mark.parametrize("name", ["tiny", "rmat12", "rmat16", "grid64", "isolated"])
@pytest.mark.parametrize("form", [0, 1, 2])  # x/deg gathers: through L1 (default and explicit), L2 only
def test_pagerank_l1(gsrb, ctx, orc, graphs, name, form):
    g = graphs[name]
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.float32)
    rc, st = dg.pagerank(out, 0.85, 50, gsrb.cfg(variant=gsrb.BAR_FANOUT, ctas_per_sm=2, threads=512,
                                                  wake_lines=4, form=form))
    gsrb.check(rc, "pagerank")
    assert st.levels == 50
    ref = orc.pagerank(g, 0.85, 50)
    got = out.download()
    assert orc.normalized_l1(got, ref) <= PR_L1_TOL
    assert np.max(np.abs(got - ref) / ref) < 1e-5


@pytest.mark.parametrize("name", ["rmat12", "grid64"])
def test_gather_probe(gsrb, ctx, graphs, name):
    dg = ctx.graph(graphs[name])
    assert dg.probe_gather(True) > 0.0 and dg.probe_gather(False) > 0.0
    assert ctx.status()[0] == 0
    dg.free()


@pytest.mark.parametrize("name", ["tiny", "rmat12", "rmat16", "grid64", "isolated"])
def test_pagerank_residual_converges_to_the_fixed_point(gsrb, ctx, orc, graphs, name):
    # the reference's push-residual algorithm: every vertex's unpropagated
    # residual ends below epsilon, so p is within about epsilon / (1 - alpha)
    # (normalised) of the FP64 fixed point p = (1 - alpha) + alpha * A^T D^-1 p
    g = graphs[name]
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.float32)
    rc, st = dg.pagerank_residual(out, 0.85, 1e-6)
    gsrb.check(rc, "pagerank_residual")
    ctx.check_status("pagerank_residual")
    ref = orc.pagerank(g, 0.85, 400)
    assert orc.normalized_l1(out.download(), ref) <= 2e-5
    assert st.levels >= 1


@pytest.mark.parametrize("shape", [(1, 64), (1, 128)])
def test_pagerank_residual_reserved_worklist_chunks(gsrb, ctx, orc, graphs, shape):
    # few warps (n >= 63 x warps): the worklist is filled through per-warp
    # reservations whose hole slots the next round skips
    g = graphs["rmat16"]
    assert 63 * (ctx.num_sms * shape[0] * shape[1] // 32) <= g.nnodes
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.float32)
    c = gsrb.cfg(variant=gsrb.BAR_FANOUT, ctas_per_sm=shape[0], threads=shape[1], wake_lines=4)
    rc, st = dg.pagerank_residual(out, 0.85, 1e-6, c=c)
    gsrb.check(rc, "pagerank_residual")
    ctx.check_status("pagerank_residual")
    assert orc.normalized_l1(out.download(), orc.pagerank(g, 0.85, 400)) <= 2e-5
    dg.free()


def test_pagerank_residual_round_cap(gsrb, ctx, graphs):
    g = graphs["rmat12"]
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.float32)
    rc, st = dg.pagerank_residual(out, 0.85, 1e-6, max_iters=3)
    gsrb.check(rc, "pagerank_residual")
    assert st.levels == 3


def test_bfs_trace_records(gsrb, ctx, orc, graphs):
    g = graphs["rmat16"]
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.int32)
    rc, st = dg.bfs(0, out, gsrb.BFS_HEURISTIC)
    gsrb.check(rc)
    tr = dg.trace()
    lv = orc.bfs(g, 0)
    sizes = np.bincount(lv[lv != 2**31 - 1])
    assert len(tr) == st.levels
    # the frontier of level L holds the vertices at level L - 1
    assert tr["nf"].tolist() == sizes[:len(tr)].tolist()
    assert set(tr["dir"].tolist()) <= {0, 1, 3}  # 3: levels run by a single CTA


def _fan_graph(gsrb):
    # directed: 0 -> 1..200000; every tenth of those -> 8 fresh vertices, the rest
    # have no out-edges, so a large push level's queue interleaves zero-degree
    # entries with short ranges (the load balancer's owner search must skip them)
    n1 = 200000
    src = [np.zeros(n1, np.uint32)]
    dst = [np.arange(1, n1 + 1, dtype=np.uint32)]
    parents = np.arange(10, n1 + 1, 10, dtype=np.uint32)
    fresh = n1 + 1 + np.arange(parents.size * 8, dtype=np.uint32)
    src.append(np.repeat(parents, 8))
    dst.append(fresh)
    n = int(fresh[-1]) + 1
    return gsrb.csr_from_edges(n, np.concatenate(src), np.concatenate(dst), symmetrize=False)


@pytest.mark.parametrize("name", ["rmat16", "grid64", "isolated", "fan"])
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("shape", [(2, 256), (1, 512), (4, 128)])
def test_bfs_load_balanced_levels_exact(gsrb, ctx, orc, graphs, name, mode, shape):
    g = _fan_graph(gsrb) if name == "fan" else graphs[name]
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.int32)
    c = gsrb.cfg(variant=gsrb.BAR_FANOUT, ctas_per_sm=shape[0], threads=shape[1], wake_lines=4)
    rc, st = dg.bfs(0, out, mode | gsrb.BFS_FLAG_LB, c)
    gsrb.check(rc, "bfs lb")
    ctx.check_status("bfs lb")
    want = orc.bfs(g, 0)
    assert np.array_equal(out.download(), want)
    assert st.edges == orc.traversed_edges(g, want)
    dg.free()


def test_bfs_load_balanced_flag_rejected_by_batches(gsrb, ctx, graphs):
    g = graphs["rmat12"]
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.int32)
    b = gsrb.Batch(ctx, [dg], gsrb.cfg(variant=gsrb.BAR_FANOUT, ctas_per_sm=1, threads=256, wake_lines=4))
    assert b.bfs([0], [out], gsrb.BFS_PUSH | gsrb.BFS_FLAG_LB) == gsrb.ERR_ARG
    b.free()
    dg.free()


def test_directed_graph_never_pulls(gsrb, ctx, orc, graphs):
    # rows are out-edges; a pull level would read them as in-edges, so on a
    # directed graph the heuristic and the policy push, and the pull-only
    # forms refuse
    g = _fan_graph(gsrb)
    dg = ctx.graph(g)
    assert not dg.symmetric and ctx.graph(graphs["rmat12"]).symmetric
    out = ctx.array(g.nnodes, np.int32)
    want = orc.bfs(g, 0)
    for mode in (gsrb.BFS_HEURISTIC, gsrb.BFS_PUSH, gsrb.BFS_TOPO):
        gsrb.check(dg.bfs(0, out, mode)[0], "bfs")
        assert np.array_equal(out.download(), want)
    assert dg.bfs(0, out, gsrb.BFS_PULL)[0] == gsrb.ERR_UNSUPPORTED
    assert dg.pagerank(ctx.array(g.nnodes, np.float32), 0.85, 5)[0] == gsrb.ERR_UNSUPPORTED
    dg.free()


@pytest.mark.parametrize("name,delta", [("rmat16", 10000), ("rmat16", 300), ("grid256", 2000)])
@pytest.mark.parametrize("shape", [(1, 64), (1, 128)])
def test_sssp_reserved_queue_chunks(gsrb, ctx, orc, graphs, name, delta, shape):
    # few warps (n >= 63 x warps), so the near queue is filled through
    # per-warp reservations with hole slots that the next round skips
    g = gsrb.grid2d(256, 256, seed=5) if name == "grid256" else graphs[name]
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.int32)
    c = gsrb.cfg(variant=gsrb.BAR_FANOUT, ctas_per_sm=shape[0], threads=shape[1], wake_lines=4)
    assert 63 * (ctx.num_sms * shape[0] * shape[1] // 32) <= g.nnodes
    rc, st = dg.sssp(0, out, delta, c)
    gsrb.check(rc, "sssp")
    ctx.check_status("sssp")
    assert np.array_equal(out.download(), orc.dijkstra(g, 0))
    dg.free()


def _head3_only(gsrb, bias):
    """Policy weights whose head 3 is the constant `bias` (hidden layers zero)
    and whose other heads say "push" and predict nothing."""
    w = np.zeros(gsrb.mlp_param_count(), np.float32)
    w[-1] = bias  # b3[3]
    return w


@pytest.mark.parametrize("bias", [-1.5, 2.0])
def test_policy_picks_the_launch(gsrb, ctx, orc, graphs, bias):
    g = graphs["rmat16"]
    dg = ctx.graph(g)
    dg.set_policy(_head3_only(gsrb, bias))
    c0 = gsrb.cfg(variant=gsrb.BAR_CCG, ctas_per_sm=2, threads=512, cluster=1)
    c1 = gsrb.cfg(variant=gsrb.BAR_FLIP, ctas_per_sm=1, threads=256, cluster=1)
    k, z = dg.policy_launch(0)
    assert z == pytest.approx(bias) and k == (1 if bias > 0 else 0)
    out = ctx.array(g.nnodes, np.int32)
    want = orc.bfs(g, 0)
    # without launch choices the default shape runs and stats.launch stays 0
    rc, st = dg.bfs(0, out, gsrb.BFS_LEARNED)
    gsrb.check(rc, "learned bfs")
    assert st.launch == 0 and np.array_equal(out.download(), want)
    dg.set_launch_choices(c0, c1)
    rc, st = dg.bfs(0, out, gsrb.BFS_LEARNED)
    gsrb.check(rc, "learned bfs, own launch")
    assert st.launch == 1 + k
    assert np.array_equal(out.download(), want)
    # an explicit cfg overrides the choice; other modes never consult it
    rc, st = dg.bfs(0, out, gsrb.BFS_LEARNED, c0)
    gsrb.check(rc)
    assert st.launch == 0
    rc, st = dg.bfs(0, out, gsrb.BFS_HEURISTIC)
    gsrb.check(rc)
    assert st.launch == 0 and np.array_equal(out.download(), want)
    dg.set_launch_choices(None, None)
    rc, st = dg.bfs(0, out, gsrb.BFS_LEARNED)
    gsrb.check(rc)
    assert st.launch == 0
    out.free()
    dg.free()


def test_policy_launch_score_matches_the_oracle_forward(gsrb, ctx, orc, graphs):
    g = graphs["grid64"]
    dg = ctx.graph(g)
    w = gsrb.mlp_init(77)
    dg.set_policy(w)
    for src in (0, 5, 1000):
        deg = int(g.row_start[src + 1] - g.row_start[src])
        x = gsrb.level_features(g.nnodes, g.nedges, 1, 1, deg, g.nnodes - 1, g.nedges - deg, 1, 0)
        want = orc.mlp_forward(w, np.asarray(x, np.float32)[None, :])[0, 3]
        k, z = dg.policy_launch(src)
        assert z == pytest.approx(want, rel=1e-4, abs=1e-5) and k == (1 if z > 0 else 0)
    dg.free()
