"""The reference's own host programs, unchanged, linked against libgsrb.

tpds22-artifact_b200/dropin/Makefile builds them from the reference sources
(the binaries travel in tpds22-artifact_b200/bin/dropin/):

* ``test_reduce``: Reduce/test_reduce.cu:8-27 calling ``reduce()``
  (Reduce/reduce.cuh:19) -- the sum of N ones, printed as "Sum:" beside
  "Correct sum:";
* ``scan``: scan/main.cu:23-83 calling ``sum_scan_blelloch()``
  (scan/scan.h:16-18) and comparing with its own ``cpu_sum_scan`` -- "Match: 1";
* ``allSyncPrims-1kernel``: Heterosync/main.cu with only its four
  ``#include "cudaLocks*.cu"`` lines (main.cu:15-18) replaced by this library's
  ``gsrb/cudaLocks.cuh`` -- every kernel of the program calls this library's
  barriers, mutexes and semaphores under the reference's names, and the
  program's own golden replay (main.cu:2987-3166) prints "PASSED!";
* ``{bfs,sssp,pr}_gg``: LONESTAR/skelapp/skel.cu.prehip (options, .gr
  loading, copy to the GPU, output) + apps/<app>/support.cu + rt/src/csr_graph.cu,
  with this library's ``gg_main`` (skel.cu.prehip:12,61) in place of the app's
  kernel file.  Levels and distances are compared with the oracle, ranks with
  the FP64 fixed point.
"""
import pathlib
import re
import subprocess

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
DROPIN = ROOT / "tpds22-artifact_b200" / "bin" / "dropin"
PROGS = ["test_reduce", "scan", "allSyncPrims-1kernel", "bfs_gg", "sssp_gg", "pr_gg"]

pytestmark = pytest.mark.skipif(not (DROPIN / "test_reduce").exists(),
                                reason="drop-in programs not built (needs the reference sources)")


def _run(prog, args, stdin=None, timeout=600):
    p = subprocess.run([str(DROPIN / prog)] + [str(a) for a in args], input=stdin, capture_output=True,
                       text=True, timeout=timeout)
    assert p.returncode == 0, p.stdout + p.stderr
    return p


@pytest.mark.parametrize("prog", PROGS)
def test_dropin_links_libgsrb(prog):
    out = subprocess.run(["ldd", str(DROPIN / prog)], capture_output=True, text=True, timeout=60).stdout
    assert "libgsrb.so" in out and "not found" not in out


@pytest.mark.parametrize("prog", ["bfs_gg", "sssp_gg", "pr_gg"])
def test_dropin_harness_usage_is_the_reference_skel(prog):
    # skel.cu.prehip:78-84 prints the usage line and exits 1 without arguments
    p = subprocess.run([str(DROPIN / prog)], capture_output=True, text=True, timeout=60)
    assert p.returncode == 1 and "usage:" in p.stderr and "graph-file" in p.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("n", [0, 1, 1000, 303_104, 1 << 24, 3_000_001])
def test_reference_reduce_driver(ctx, n):
    p = _run("test_reduce", [n, 256])
    assert f"Sum: {n}\n" in p.stdout and f"Correct sum: {n}\n" in p.stdout
    assert "time (ms) is" in p.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("tpb", [32, 100, 1024])
def test_reference_reduce_driver_block_sizes(ctx, tpb):
    # block sizes that are not a CTA size the library uses fall back to its default
    p = _run("test_reduce", [123_457, tpb])
    assert "Sum: 123457\n" in p.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 64, 65, 4097, 303_104, 1 << 20, (1 << 24) + 3])
def test_reference_scan_driver(ctx, n):
    p = _run("scan", [n])
    assert f"h_in size: {n}" in p.stdout
    assert "Match: 1" in p.stdout, p.stdout[-2000:]


def _read_pairs(path, n, dtype):
    out = np.zeros(n, dtype)
    seen = np.zeros(n, bool)
    for line in pathlib.Path(path).read_text().splitlines():
        i, v = line.split()[:2]
        out[int(i)] = np.iinfo(np.int32).max if v == "INF" else dtype(float(v)) if dtype is np.float64 else int(v)
        seen[int(i)] = True
    assert seen.all()
    return out


@pytest.fixture(scope="module")
def dropin_graphs(gsrb, tmp_path_factory):
    d = tmp_path_factory.mktemp("dropin_gr")
    gs = {"tiny": gsrb.Graph.read_gr(ROOT / "tests" / "golden" / "tiny.gr"),
          "rmat12": gsrb.rmat(12, 16, seed=31),
          "grid": gsrb.grid2d(64, 48, seed=5)}
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
@pytest.mark.parametrize("name", ["tiny", "rmat12", "grid", "split"])
@pytest.mark.parametrize("lb", [False, True])
def test_reference_skel_bfs(ctx, orc, dropin_graphs, tmp_path, name, lb):
    path, g = dropin_graphs[name]
    out = tmp_path / "bfs.txt"
    args = (["-l"] if lb else []) + ["-s", "0", "-o", out, path]
    p = _run("bfs_gg", args, stdin="2\n")
    assert "Enter Block factor" in p.stdout and "Kernel time (ms)" in p.stdout
    assert np.array_equal(_read_pairs(out, g.nnodes, np.int64).astype(np.int32), orc.bfs(g, 0))


@pytest.mark.gpu
@pytest.mark.parametrize("name,delta", [("tiny", None), ("rmat12", None), ("grid", 64), ("split", 1)])
def test_reference_skel_sssp(ctx, orc, dropin_graphs, tmp_path, name, delta):
    path, g = dropin_graphs[name]
    out = tmp_path / "sssp.txt"
    args = (["-d", delta] if delta else []) + ["-s", "0", "-o", out, path]
    p = _run("sssp_gg", args, stdin="1\n")
    assert f"delta: {delta or 10000}" in p.stdout and "iterations:" in p.stdout
    assert np.array_equal(_read_pairs(out, g.nnodes, np.int64).astype(np.int32), orc.dijkstra(g, 0))


@pytest.mark.gpu
def test_reference_skel_pr(ctx, orc, dropin_graphs, tmp_path):
    path, g = dropin_graphs["rmat12"]
    out = tmp_path / "pr.txt"
    p = _run("pr_gg", ["-o", out, path], stdin="2\n")
    it = re.search(r"PR took (\d+) iterations", p.stdout)
    assert it and int(it.group(1)) > 0
    assert re.search(r"sum: [0-9.]+ \(%d\)" % g.nnodes, p.stdout)
    r = _read_pairs(out, g.nnodes, np.float64)
    ref = orc.pagerank(g, 0.85, 400)
    # push-residual to epsilon 1e-6 against the FP64 fixed point; "%f" keeps six decimals
    tol = 2e-5 + 5e-7 * g.nnodes / ref.sum()
    assert np.abs(r - ref).sum() / ref.sum() <= tol


@pytest.mark.gpu
def test_reference_skel_quiet(ctx, dropin_graphs, tmp_path):
    path, _ = dropin_graphs["tiny"]
    out = tmp_path / "none.txt"
    _run("bfs_gg", ["-q", "-o", out, path], stdin="1\n")
    assert not out.exists()


# the reference program's syncPrim names (Heterosync/main.cu:2478-2535)
HETEROSYNC_PRIMS = [
    "atomicTreeBarrUniq", "atomicTreeBarrUniqLocalExch", "lfTreeBarrUniq", "lfTreeBarrUniqLocalExch",
    "spinMutex", "spinMutexEBO", "sleepMutex", "faMutex",
    "spinSem1", "spinSem2", "spinSem10", "spinSem120", "spinSemEBO1", "spinSemEBO2", "spinSemEBO10",
    "spinSemEBO120", "PRspinSem1", "PRspinSem2", "PRspinSem10", "PRspinSem120",
    "spinMutexUniq", "spinMutexEBOUniq", "sleepMutexUniq", "faMutexUniq",
    "spinSemUniq1", "spinSemUniq2", "spinSemUniq10", "spinSemUniq120", "spinSemEBOUniq1", "spinSemEBOUniq2",
    "spinSemEBOUniq10", "spinSemEBOUniq120",
    "atomicTreeBarrUniqSRB", "atomicTreeBarrUniqLocalExchSRB", "atomicTreeBarrUniqNaiveSRB",
    "atomicTreeBarrUniqLocalExchNaiveSRB", "atomicTreeBarrUniqNaiveAllSRB",
    "atomicTreeBarrUniqLocalExchNaiveAllSRB", "atomicTreeBarrUniqHybridSRB",
    "atomicTreeBarrUniqLocalExchHybridSRB", "atomicTreeBarrUniqCCG", "atomicTreeBarrUniqLocalExchCCG"]


def test_dropin_heterosync_source_differs_only_in_includes():
    # the compiled copy is the reference's main.cu with the include lines swapped
    src = ROOT / "tpds22-artifact_b200" / "build" / "dropin" / "heterosync" / "main.cu"
    if not src.exists():
        pytest.skip("scratch copy not present (built elsewhere)")
    text = src.read_text().splitlines()
    assert sum("gsrb/cudaLocks.cuh" in line for line in text) == 1
    assert not any(line.startswith('#include "cudaLocks') for line in text)


@pytest.mark.gpu
@pytest.mark.parametrize("prim", HETEROSYNC_PRIMS)
def test_reference_heterosync_program_on_library(ctx, prim):
    # 2 CTAs of 32 threads per SM (co-resident), 10 loads/stores, 2 iterations;
    # the program launches its kernel 10 times and checks its storage array
    # against its own golden replay
    p = _run("allSyncPrims-1kernel", [prim, 10, 2 * ctx.num_sms, 2], timeout=300)
    assert "PASSED!" in p.stdout, (p.stdout + p.stderr)[-3000:]
    assert re.search(r"elapsed time: [0-9.]+ ms, average: [0-9.]+ ms", p.stdout)
