"""The Lonestar harness binaries (bin/{bfs,sssp,pr}_{gsrb,gcpusrb,ccg}).

They keep the reference skel harness's command line, block-factor prompt and
output format (LONESTAR/skelapp/skel.cu.prehip:45-130,
LONESTAR/apps/bfs/support.cu:27-45, LONESTAR/apps/pr/support.cu:45-98); the GPU
tests run them on .gr files and compare the written levels / distances / ranks
with the oracle.
"""
import pathlib
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
BIN = ROOT / "tpds22-artifact_b200" / "bin"
APPS = [f"{a}_{v}" for a in ("bfs", "sssp", "pr") for v in ("gsrb", "gcpusrb", "ccg")]


@pytest.mark.parametrize("app", APPS)
def test_app_usage(app):
    p = subprocess.run([str(BIN / app)], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1
    assert "usage:" in p.stderr and "graph-file" in p.stderr
    if app.startswith("sssp"):
        assert "-d delta" in p.stderr
    if app.startswith("pr"):
        assert "-x max_iterations" in p.stderr


def test_app_bad_option():
    p = subprocess.run([str(BIN / "bfs_gsrb"), "-Z", "x.gr"], capture_output=True, text=True, timeout=60)
    assert p.returncode != 0 and "usage:" in p.stderr


def _run(app, args, block_factor="2"):
    p = subprocess.run([str(BIN / app)] + args, input=f"{block_factor}\n", capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "Enter Block factor" in p.stdout
    return p


def _read_levels(path, n):
    out = np.full(n, -1, dtype=np.int64)
    for line in pathlib.Path(path).read_text().splitlines():
        i, v = line.split()
        out[int(i)] = np.iinfo(np.int32).max if v == "INF" else int(v)
    assert (out >= 0).all()
    return out.astype(np.int32)


@pytest.fixture(scope="module")
def gr_files(gsrb, tmp_path_factory):
    d = tmp_path_factory.mktemp("gr")
    gs = {"tiny": gsrb.Graph.read_gr(ROOT / "tests" / "golden" / "tiny.gr"),
          "rmat12": gsrb.rmat(12, 16, seed=31),
          "grid": gsrb.grid2d(64, 48, seed=5)}
    # an extra disconnected piece so INF lines appear
    src = np.array([0, 1, 2, 10, 11], np.uint32)
    dst = np.array([1, 2, 3, 11, 12], np.uint32)
    gs["split"] = gsrb.csr_from_edges(20, src, dst)
    files = {}
    for k, g in gs.items():
        p = d / f"{k}.gr"
        g.write_gr(p, with_weights=True)
        files[k] = (p, g)
    return files


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["gsrb", "gcpusrb", "ccg"])
@pytest.mark.parametrize("name", ["tiny", "rmat12", "grid", "split"])
def test_bfs_app_matches_oracle(ctx, orc, gr_files, tmp_path, variant, name):
    path, g = gr_files[name]
    out = tmp_path / "levels.txt"
    p = _run(f"bfs_{variant}", ["-s", "0", "-o", str(out), str(path)])
    assert "Kernel time (ms)" in p.stdout
    assert np.array_equal(_read_levels(out, g.nnodes), orc.bfs(g, 0))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["push", "heuristic"])
def test_bfs_app_load_balanced(ctx, orc, gr_files, tmp_path, mode):
    # -l: the reference's load-balanced expansion (GSRB_BFS_FLAG_LB)
    path, g = gr_files["rmat12"]
    out = tmp_path / "levels.txt"
    _run("bfs_gsrb", ["-l", "-s", "3", "-m", mode, "-o", str(out), str(path)], block_factor="1")
    assert np.array_equal(_read_levels(out, g.nnodes), orc.bfs(g, 3))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["push", "pull", "topo", "learned"])
def test_bfs_app_modes(gsrb, ctx, orc, gr_files, tmp_path, mode):
    path, g = gr_files["rmat12"]
    out = tmp_path / "levels.txt"
    extra = []
    if mode == "learned":
        # any weights: the policy changes the schedule, never the levels
        wfile = tmp_path / "policy.f32"
        gsrb.mlp_init(7).astype(np.float32).tofile(wfile)
        extra = ["-P", str(wfile)]
    _run("bfs_gsrb", ["-s", "3", "-m", mode] + extra + ["-o", str(out), str(path)], block_factor="1")
    assert np.array_equal(_read_levels(out, g.nnodes), orc.bfs(g, 3))


@pytest.mark.gpu
def test_bfs_app_learned_needs_policy(ctx, gr_files):
    path, _ = gr_files["rmat12"]
    p = subprocess.run([str(BIN / "bfs_gsrb"), "-m", "learned", str(path)], input="1\n", capture_output=True,
                       text=True, timeout=120)
    assert p.returncode != 0 and "gsrb_bfs" in p.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["gsrb", "gcpusrb", "ccg"])
@pytest.mark.parametrize("name,delta", [("rmat12", 10000), ("grid", 64), ("split", 1)])
def test_sssp_app_matches_oracle(ctx, orc, gr_files, tmp_path, variant, name, delta):
    path, g = gr_files[name]
    out = tmp_path / "dist.txt"
    p = _run(f"sssp_{variant}", ["-d", str(delta), "-s", "0", "-o", str(out), str(path)])
    assert f"delta: {delta}" in p.stdout and "iterations:" in p.stdout
    assert np.array_equal(_read_levels(out, g.nnodes), orc.dijkstra(g, 0))


def _read_ranks(path, n):
    r = np.zeros(n, np.float64)
    for line in path.read_text().splitlines():
        i, v = line.split()
        r[int(i)] = float(v)
    return r


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["gsrb", "ccg"])
def test_pr_app_pull_matches_oracle(ctx, orc, gr_files, tmp_path, variant):
    path, g = gr_files["rmat12"]
    out = tmp_path / "ranks.txt"
    p = _run(f"pr_{variant}", ["-u", "-x", "50", "-o", str(out), str(path)])
    assert "PR took 50 iterations" in p.stdout and "sum:" in p.stdout
    r = _read_ranks(out, g.nnodes)
    ref = orc.pagerank(g, 0.85, 50)
    # "%f" keeps 6 decimals: allow the printing rounding on top of the 1e-6 bound
    tol = 1e-6 + 5e-7 * g.nnodes / ref.sum()
    assert np.abs(r - ref).sum() / ref.sum() <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["gsrb", "gcpusrb"])
def test_pr_app_default_is_the_reference_residual_algorithm(ctx, orc, gr_files, tmp_path, variant):
    path, g = gr_files["rmat12"]
    out = tmp_path / "ranks.txt"
    p = _run(f"pr_{variant}", ["-o", str(out), str(path)])
    assert "PR took" in p.stdout and "sum:" in p.stdout
    r = _read_ranks(out, g.nnodes)
    ref = orc.pagerank(g, 0.85, 400)
    tol = 2e-5 + 5e-7 * g.nnodes / ref.sum()
    assert np.abs(r - ref).sum() / ref.sum() <= tol


@pytest.mark.gpu
def test_app_quiet_writes_nothing(ctx, gr_files, tmp_path):
    path, _ = gr_files["tiny"]
    out = tmp_path / "none.txt"
    _run("bfs_gsrb", ["-q", "-o", str(out), str(path)])
    assert not out.exists()


@pytest.mark.gpu
def test_app_rejects_bad_start(ctx, gr_files):
    path, g = gr_files["tiny"]
    p = subprocess.run([str(BIN / "bfs_gsrb"), "-s", str(g.nnodes + 5), str(path)], input="2\n",
                       capture_output=True, text=True, timeout=120)
    assert p.returncode != 0 and "out of range" in p.stderr
