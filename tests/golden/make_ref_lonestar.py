"""Golden outputs of the reference's own Lonestar programs, for graph parity.

The reference has no CPU BFS / SSSP / PageRank; its results come from its GPU
programs.  This script runs them -- oracle/_ref/lonestar/{bfs,sssp,pr}_ccg, the
reference's LONESTAR/apps/<app>/kernel_ccg.cu with its skel harness, built for
sm_100a by baseline/build.sh -- on small seeded graphs written as .gr v1,
and stores what they print (LONESTAR/apps/bfs/support.cu:27-46 "%d %d" /
"%d INF" lines, sssp/support.cu:35-52, pr/support.cu:45-98) in one .npz:

* ``<graph>/fingerprint``: n, m and a hash of row_start / edge_dst / edge_data,
  so a test that rebuilds the graph from its seed knows it is the same input;
* ``<graph>/bfs_s<src>``: int32 levels (INT_MAX for INF);
* ``<graph>/sssp_s<src>_d<delta>``: int32 distances;
* ``<graph>/pr``: float32 ranks of the push-residual PageRank (FP32 atomics:
  not deterministic run to run; tests compare it within a tolerance).

The cooperative-groups forms are used because their launch is refused, not
hung, when the grid cannot be co-resident.  Needs a GPU; run on a B200 with

    python tests/golden/make_ref_lonestar.py gpurun_out/ref_lonestar_golden.npz

and commit the result as tests/golden/ref_lonestar_golden.npz.
"""
import hashlib
import pathlib
import subprocess
import sys
import tempfile

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
REF = ROOT / "baseline" / "_ref" / "lonestar"
sys.path.insert(0, str(ROOT / "tests"))


def binding():
    import conftest  # noqa: F401  (builds the library if needed)
    return conftest._load_binding()


def graphs(g):
    """The golden graphs, rebuilt the same way by the parity tests."""
    src = np.array([0, 1, 2, 10, 11], np.uint32)
    dst = np.array([1, 2, 3, 11, 12], np.uint32)
    rs = np.random.default_rng(9)
    dsrc = rs.integers(0, 600, 4000).astype(np.uint32)
    ddst = rs.integers(0, 600, 4000).astype(np.uint32)
    return {
        "tiny": g.Graph.read_gr(ROOT / "tests" / "golden" / "tiny.gr"),
        "split": g.csr_from_edges(20, src, dst),
        "rmat12": g.rmat(12, 16, seed=31),
        "rmat14": g.rmat(14, 16, seed=77),
        "grid": g.grid2d(64, 48, seed=5),
        "directed": g.csr_from_edges(600, dsrc, ddst, symmetrize=False, weight_seed=3),
    }


# (graph, BFS sources, SSSP (source, delta) pairs, PageRank?)
PLAN = {
    "tiny": ([0, 2], [(0, 10000)], True),
    "split": ([0, 11], [(0, 10000), (0, 1)], True),
    "rmat12": ([0, 3], [(0, 10000), (3, 64)], True),
    "rmat14": ([0], [(0, 10000), (0, 32)], True),
    "grid": ([0, 1000], [(0, 10000), (0, 64)], True),
    "directed": ([0, 5], [(0, 10000)], True),
}


def fingerprint(gr):
    h = hashlib.sha256()
    for a in (gr.row_start, gr.edge_dst, gr.edge_data):
        h.update(np.ascontiguousarray(a).tobytes())
    return np.frombuffer(h.digest()[:16], np.uint8).copy(), gr.nnodes, int(gr.edge_dst.size)


def read_pairs(text, n, floats=False):
    out = np.zeros(n, np.float32 if floats else np.int32)
    seen = np.zeros(n, bool)
    for line in text.splitlines():
        parts = line.split()
        i = int(parts[0])
        v = parts[1]
        out[i] = np.iinfo(np.int32).max if v == "INF" else (float(v) if floats else int(v))
        seen[i] = True
    if not seen.all():
        raise RuntimeError(f"output covers {seen.sum()} of {n} vertices")
    return out


def run(prog, args, path, tmp):
    out = tmp / "out.txt"
    cmd = [str(REF / prog)] + [str(a) for a in args] + ["-o", str(out), str(path)]
    p = subprocess.run(cmd, input="2\n", capture_output=True, text=True, timeout=300)
    if p.returncode != 0:
        raise RuntimeError(f"{cmd}: rc {p.returncode}\n{p.stdout}\n{p.stderr}")
    return out.read_text(), p.stdout


def main(dest):
    g = binding()
    res = {}
    log = []
    with tempfile.TemporaryDirectory() as td:
        tmp = pathlib.Path(td)
        for name, gr in graphs(g).items():
            bfs_srcs, sssp_runs, do_pr = PLAN[name]
            path = tmp / f"{name}.gr"
            gr.write_gr(path, with_weights=True)
            fp, n, m = fingerprint(gr)
            res[f"{name}/fingerprint"] = fp
            res[f"{name}/nm"] = np.array([n, m], np.int64)
            for s in bfs_srcs:
                text, so = run("bfs_ccg", ["-s", s], path, tmp)
                res[f"{name}/bfs_s{s}"] = read_pairs(text, n)
                log.append(f"{name} bfs s{s}: {so.strip().splitlines()[-2:]}")
            for s, d in sssp_runs:
                text, so = run("sssp_ccg", ["-s", s, "-d", d], path, tmp)
                res[f"{name}/sssp_s{s}_d{d}"] = read_pairs(text, n)
                log.append(f"{name} sssp s{s} d{d}: {so.strip().splitlines()[-2:]}")
            if do_pr:
                text, so = run("pr_ccg", [], path, tmp)
                res[f"{name}/pr"] = read_pairs(text, n, floats=True)
                log.append(f"{name} pr: {so.strip().splitlines()[-2:]}")
    np.savez_compressed(dest, **res)
    print("\n".join(log))
    print(f"wrote {len(res)} arrays to {dest}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "ref_lonestar_golden.npz")
