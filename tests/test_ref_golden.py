"""Graph parity pinned on the reference's own outputs.

tests/golden/ref_lonestar_golden.npz holds what the reference's Lonestar
programs (LONESTAR/apps/{bfs,sssp,pr}/kernel_ccg.cu with the reference's skel
harness, built for sm_100a by baseline/build.sh) printed for six seeded graphs
(tests/golden/make_ref_lonestar.py made it on a B200).  The CPU tests pin the
oracle to it: BFS levels and SSSP distances bit-exact, PageRank within the
push-residual tolerance.  The GPU tests hold this library's traversals, and
the reference's skel harness running this library's gg_main, to the same
outputs directly.
"""
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "tests" / "golden"))
import make_ref_lonestar as golden  # noqa: E402

GOLD = np.load(ROOT / "tests" / "golden" / "ref_lonestar_golden.npz")
NAMES = list(golden.PLAN)


@pytest.fixture(scope="module")
def graphs(gsrb):
    return golden.graphs(gsrb)


def _keys(name, kind):
    return [k for k in GOLD.files if k.startswith(f"{name}/{kind}")]


def _pr_tol(ref):
    # epsilon-converged push residuals plus the reference's "%f" (six decimals) output
    return 2e-5 + 5e-7 * ref.size / ref.sum()


@pytest.mark.parametrize("name", NAMES)
def test_golden_graph_is_the_same_input(graphs, name):
    fp, n, m = golden.fingerprint(graphs[name])
    assert np.array_equal(fp, GOLD[f"{name}/fingerprint"])
    assert [n, m] == GOLD[f"{name}/nm"].tolist()


@pytest.mark.parametrize("name", NAMES)
def test_oracle_bfs_equals_reference(orc, graphs, name):
    for k in _keys(name, "bfs_s"):
        src = int(k.split("bfs_s")[1])
        assert np.array_equal(orc.bfs(graphs[name], src), GOLD[k]), k


@pytest.mark.parametrize("name", NAMES)
def test_oracle_dijkstra_equals_reference(orc, graphs, name):
    for k in _keys(name, "sssp_s"):
        src = int(k.split("sssp_s")[1].split("_")[0])
        assert np.array_equal(orc.dijkstra(graphs[name], src), GOLD[k]), k


@pytest.mark.parametrize("name", NAMES)
def test_oracle_pagerank_fixed_point_matches_reference(orc, graphs, name):
    ref = orc.pagerank_push(graphs[name], 0.85, 400)
    got = GOLD[f"{name}/pr"].astype(np.float64)
    assert np.abs(got - ref).sum() / ref.sum() <= _pr_tol(ref)


def test_oracle_pull_form_differs_on_the_directed_graph(orc, graphs):
    # the pull restatement reads rows as in-edges: right only for symmetric graphs
    g = graphs["directed"]
    pull, push = orc.pagerank(g, 0.85, 400), orc.pagerank_push(g, 0.85, 400)
    assert np.abs(pull - push).sum() / push.sum() > 1e-2
    s = graphs["rmat12"]
    assert np.abs(orc.pagerank(s, 0.85, 100) - orc.pagerank_push(s, 0.85, 100)).max() < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_library_traversals_equal_reference(gsrb, ctx, graphs, name):
    g = graphs[name]
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.int32)
    for k in _keys(name, "bfs_s"):
        src = int(k.split("bfs_s")[1])
        for mode in (gsrb.BFS_PUSH, gsrb.BFS_HEURISTIC, gsrb.BFS_PUSH | gsrb.BFS_FLAG_LB):
            rc, _ = dg.bfs(src, out, mode)
            gsrb.check(rc, "bfs")
            assert np.array_equal(out.download(), GOLD[k]), f"{k} mode {mode}"
    for k in _keys(name, "sssp_s"):
        src, delta = (int(x) for x in k.split("sssp_s")[1].split("_d"))
        rc, _ = dg.sssp(src, out, delta)
        gsrb.check(rc, "sssp")
        assert np.array_equal(out.download(), GOLD[k]), k
    r = ctx.array(g.nnodes, np.float32)
    rc, _ = dg.pagerank_residual(r, 0.85, 1e-6, 2**31 - 1)
    gsrb.check(rc, "pagerank_residual")
    ref = GOLD[f"{name}/pr"].astype(np.float64)
    assert np.abs(r.download().astype(np.float64) - ref).sum() / ref.sum() <= 2 * _pr_tol(ref)
    dg.free()


DROPIN = ROOT / "tpds22-artifact_b200" / "bin" / "dropin"


@pytest.mark.gpu
@pytest.mark.skipif(not (DROPIN / "bfs_gg").exists(), reason="drop-in harness not built")
@pytest.mark.parametrize("name", ["tiny", "rmat12", "grid", "directed"])
def test_reference_harness_on_library_equals_reference(ctx, graphs, tmp_path, name):
    g = graphs[name]
    path = tmp_path / f"{name}.gr"
    g.write_gr(path, with_weights=True)
    for app, kind in (("bfs_gg", "bfs_s"), ("sssp_gg", "sssp_s")):
        for k in _keys(name, kind):
            tail = k.split(kind)[1]
            args = ["-s", tail.split("_")[0]] + (["-d", tail.split("_d")[1]] if "_d" in tail else [])
            out = tmp_path / "out.txt"
            p = subprocess.run([str(DROPIN / app)] + args + ["-o", str(out), str(path)], input="2\n",
                               capture_output=True, text=True, timeout=300)
            assert p.returncode == 0, p.stdout + p.stderr
            got = golden.read_pairs(out.read_text(), g.nnodes)
            assert np.array_equal(got, GOLD[k]), f"{app} {k}"
