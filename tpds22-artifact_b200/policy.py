"""The learned per-level policy of the BFS level loop: trace collection, labels,
training on the GPU (gsrb_mlp_train) and evaluation helpers.

The plain traversals emit one 48-byte record per level (gsrb_graph_trace):
frontier size and out-edges, unvisited vertices and their edges, and the
%globaltimer stamp at the start of the level.  Running the same BFS with the
worklist push, the pull and the topology push gives, for every level, the time
each direction took on the same frontier (the level sets do not depend on the
direction).  Those times label each level:

    head 0: pull faster than worklist push     (BCE)
    head 1: topology push faster than worklist push (BCE)
    (both weighted by |log2 of the time ratio|: the loss follows the cost of a
    wrong choice, not the count of levels)
    head 2: log2(1 + size of the next frontier) (squared error)
    head 3: log2(t0 / t1), the heuristic traversal's time under launch
            configuration 0 over that under configuration 1 (squared error;
            gsrb_graph_set_launch_choices).  The library reads it on the first
            level's features only, whose frontier is the source, so it is
            trained on extra rows: the first-level features of a sample of
            sources (their degrees), all carrying the graph's label.

Features are computed by gsrb_level_features, the host twin of the function the
traversal kernel evaluates on the device.  The policy changes only which
direction a level runs in, never the levels; it falls back to the fixed
heuristic for the rest of a traversal once its next-frontier prediction misses
by more than 2x.
"""
from __future__ import annotations

import numpy as np

INF = 2**31 - 1


def _g():
    import sys
    return sys.modules["gsrb_b200"]


def level_times(trace: np.ndarray, total_ms: float | None = None) -> np.ndarray:
    """Duration of each level (ns) from consecutive start stamps; the last
    level has no successor stamp and gets NaN."""
    t = trace["t_ns"].astype(np.float64)
    d = np.full(len(t), np.nan)
    if len(t) > 1:
        d[:-1] = np.diff(t)
    return d


TOPO_MARGIN = 0.8
# level rows of one graph count as at most LEVEL_CAP rows: a mesh has thousands
# of near-identical levels and an R-MAT graph six to ten, and without the cap
# the meshes decide the fit of every head (one added 4.7 M-vertex mesh once
# made the next-frontier head miss R-MAT's second level by more than 2x, so
# every R-MAT traversal fell back to the heuristic)
LEVEL_CAP = 64
# weight of one launch row, and the sources sampled per graph for them (a few
# rows per graph against thousands of level rows)
LAUNCH_WEIGHT = 10.0
LAUNCH_SOURCES = 16


def launch_candidates():
    """The two launch configurations head 3 chooses between: the call-wide
    default shape (2 x 512 threads per SM, grid.sync barrier), which suits
    power-law graphs whose few levels carry millions of edges, and one
    256-thread CTA per SM with the split-counter barrier, which suits meshes
    whose thousands of thin levels are barrier-bound (148 participants per
    barrier; on the 2048^2 grid 27.5 ms against 30.4 at 2 x 256)."""
    g = _g()
    return (g.cfg(variant=g.BAR_CCG, ctas_per_sm=2, threads=512, cluster=1),
            g.cfg(variant=g.BAR_FLIP, ctas_per_sm=1, threads=256, cluster=1))


def _weight(t_a: float, t_b: float) -> float:
    """Cost-sensitive sample weight: |log2(t_a / t_b)| clipped to [0.05, 4].
    A level where the two directions take about the same time hardly matters;
    one where the wrong choice costs 10x dominates the loss."""
    r = abs(np.log2(max(t_a, 1.0) / max(t_b, 1.0)))
    return float(min(4.0, max(0.05, r)))


def launch_times(ctx, dgraph, cfgs, src: int = 0, reps: int = 2) -> np.ndarray:
    """Kernel time (ms, fastest of `reps`) of the heuristic BFS from src under
    each launch configuration."""
    g = _g()
    out = ctx.array(dgraph.n, np.int32)
    t = np.zeros(len(cfgs))
    for k, c in enumerate(cfgs):
        best = np.inf
        for _ in range(reps):
            rc, st = dgraph.bfs(src, out, g.BFS_HEURISTIC, c)
            g.check(rc, "bfs (launch labels)")
            best = min(best, float(st.kernel_ms))
        t[k] = best
    out.free()
    return t


def collect_traces(ctx, dgraph, src: int = 0, reps: int = 1, launch_cfgs=None) -> dict:
    """Raw material of one graph: the per-level trace of the worklist push, the
    pull and the topology push traversals (the fastest of `reps` runs per
    level), the graph's size and, with launch_cfgs, the heuristic traversal's
    time under each of the two launch configurations.  Storable with
    save_traces."""
    g = _g()
    rec = {"n": int(dgraph.n), "m": int(dgraph.m), "src": int(src)}
    if launch_cfgs is not None:
        rec["launch_ms"] = launch_times(ctx, dgraph, launch_cfgs, src, max(reps, 2))
        deg = dgraph.host.degrees()
        rng = np.random.default_rng(rec["n"] * 1_000_003 + rec["m"])
        pick = rng.integers(0, rec["n"], LAUNCH_SOURCES - 1)
        rec["launch_degs"] = np.concatenate([[deg[src]], deg[pick]]).astype(np.int64)
    out = ctx.array(dgraph.n, np.int32)
    for name, mode in (("push", g.BFS_PUSH), ("pull", g.BFS_PULL), ("topo", g.BFS_TOPO)):
        best = None
        for _ in range(reps):
            rc, st = dgraph.bfs(src, out, mode)
            g.check(rc, "bfs (trace collection)")
            tr = dgraph.trace()
            d = level_times(tr)
            best = d if best is None else np.fmin(best, d)
        rec[name] = tr
        rec[name + "_ns"] = best
    out.free()
    return rec


def features_labels(rec: dict):
    """Per-level features, labels and cost-sensitive masks from one graph's
    traces (collect_traces or load_traces)."""
    g = _g()
    n, m = rec["n"], rec["m"]
    tr = rec["push"]
    t_push, t_pull, t_topo = rec["push_ns"], rec["pull_ns"], rec["topo_ns"]
    L = len(tr)
    X = np.zeros((L, 12), np.float32)
    Y = np.zeros((L, 4), np.float32)
    M = np.zeros((L, 4), np.float32)
    prev_nf, prev_dir = 1, 0
    for i in range(L):
        r = tr[i]
        X[i] = g.level_features(n, m, int(r["level"]), int(r["nf"]), int(r["mf"]), int(r["nu"]), int(r["mu"]),
                                prev_nf, prev_dir)
        prev_nf = int(r["nf"])
        if i < len(t_pull) and np.isfinite(t_push[i]) and np.isfinite(t_pull[i]) and i > 0:
            Y[i, 0] = 1.0 if t_pull[i] < t_push[i] else 0.0
            M[i, 0] = _weight(t_push[i], t_pull[i])
        if i < len(t_topo) and np.isfinite(t_push[i]) and np.isfinite(t_topo[i]):
            # the topology push scans every vertex: label it only where it wins
            # clearly (by 20 %), so that near-ties teach the safe worklist push
            Y[i, 1] = 1.0 if t_topo[i] < TOPO_MARGIN * t_push[i] else 0.0
            M[i, 1] = _weight(t_push[i], t_topo[i])
        nxt = int(tr[i + 1]["nf"]) if i + 1 < L else 0
        Y[i, 2] = np.log2(1.0 + nxt)
        M[i, 2] = 1.0
        prev_dir = 1 if Y[i, 0] > 0.5 and M[i, 0] > 0 else 0
    if L > LEVEL_CAP:
        M[:, :3] *= LEVEL_CAP / L
    if rec.get("launch_ms") is not None:
        # launch rows: the first level's features from each sampled source
        t0, t1 = (max(float(x), 1e-6) for x in rec["launch_ms"])
        degs = rec.get("launch_degs")
        degs = [int(tr[0]["mf"])] if degs is None else [int(d) for d in degs]
        Xl = np.stack([g.level_features(n, m, 1, 1, d, n - 1, m - d, 1, 0) for d in degs]).astype(np.float32)
        Yl = np.zeros((len(degs), 4), np.float32)
        Ml = np.zeros((len(degs), 4), np.float32)
        Yl[:, 3] = float(np.clip(np.log2(t0 / t1), -4.0, 4.0))
        Ml[:, 3] = LAUNCH_WEIGHT
        X, Y, M = np.concatenate([X, Xl]), np.concatenate([Y, Yl]), np.concatenate([M, Ml])
    return X, Y, M


def collect(ctx, dgraph, src: int = 0, reps: int = 1, launch_cfgs=None):
    """Per-level features, labels and masks of one graph from three traversals
    (and two more per launch configuration with launch_cfgs)."""
    rec = collect_traces(ctx, dgraph, src, reps, launch_cfgs)
    X, Y, M = features_labels(rec)
    return X, Y, M, {"push": rec["push_ns"], "pull": rec["pull_ns"], "topo": rec["topo_ns"],
                     "launch_ms": rec.get("launch_ms")}


def save_traces(path, recs) -> None:
    """Store the traces of several graphs in one .npz (offline training and
    replay, in the spirit of the reference's Worklist::save/load,
    LONESTAR/rt/include/worklist.h.prehip:183-220)."""
    arrays = {"count": np.array([len(recs)], np.int64)}
    for k, rec in enumerate(recs):
        arrays[f"g{k}_meta"] = np.array([rec["n"], rec["m"], rec["src"]], np.int64)
        if rec.get("launch_ms") is not None:
            arrays[f"g{k}_launch_ms"] = np.asarray(rec["launch_ms"], np.float64)
        if rec.get("launch_degs") is not None:
            arrays[f"g{k}_launch_degs"] = np.asarray(rec["launch_degs"], np.int64)
        for name in ("push", "pull", "topo"):
            arrays[f"g{k}_{name}"] = rec[name]
            arrays[f"g{k}_{name}_ns"] = np.asarray(rec[name + "_ns"], np.float64)
    np.savez_compressed(path, **arrays)


def load_traces(path) -> list:
    z = np.load(path)
    recs = []
    for k in range(int(z["count"][0])):
        n, m, src = (int(x) for x in z[f"g{k}_meta"])
        rec = {"n": n, "m": m, "src": src}
        for key in ("launch_ms", "launch_degs"):
            if f"g{k}_{key}" in z:
                rec[key] = z[f"g{k}_{key}"]
        for name in ("push", "pull", "topo"):
            rec[name] = z[f"g{k}_{name}"]
            rec[name + "_ns"] = z[f"g{k}_{name}_ns"]
        recs.append(rec)
    return recs


def dataset(recs):
    """Stacked (X, Y, M) of many graphs' traces."""
    parts = [features_labels(r) for r in recs]
    return tuple(np.concatenate([p[i] for p in parts]) for i in range(3))


def train(ctx, X, Y, M, steps: int = 3000, lr: float = 3e-3, seed: int = 2022):
    """Adam on the GPU (one persistent launch); returns (params, loss history)."""
    g = _g()
    # normalise the regression target's weight so it does not dominate the loss
    M = M.copy()
    M[:, 2] *= 0.05
    p0 = g.mlp_init(seed)
    return g.mlp_train(ctx, p0, X, Y, M, steps=steps, lr=lr)


def accuracy(ctx, params, X, Y, M):
    g = _g()
    out = g.mlp_forward(ctx, params, X)
    res = {}
    for h in (0, 1):
        sel = M[:, h] > 0
        if sel.any():
            res[f"head{h}_acc"] = float(np.mean((out[sel, h] > 0) == (Y[sel, h] > 0.5)))
    sel = M[:, 2] > 0
    if sel.any():
        res["head2_within_2x"] = float(np.mean(np.abs(out[sel, 2] - Y[sel, 2]) <= 1.0))
    sel = M[:, 3] > 0
    if sel.any():
        # launch choice: the sign of head 3 against the sign of the measured ratio
        res["head3_launch_acc"] = float(np.mean((out[sel, 3] > 0) == (Y[sel, 3] > 0)))
    return res


def save(path, params: np.ndarray):
    np.save(path, np.asarray(params, dtype=np.float32))


def load(path) -> np.ndarray:
    return np.load(path).astype(np.float32)


# ---------------------------------------------------------------- SSSP policy
# The SSSP policy uses the same network layout with its own weights, evaluated
# on the host once per traversal (gsrb_graph_sssp_plan):
#   head 2: log2(bucket width / mean edge weight)   (squared error)
#   head 3: log2(t0 / t1) over the two launch configurations (squared error)
# Labels come from timed SSSP runs of each training graph: every width of
# SSSP_DELTAS under both launch configurations.  Heads 0-1 are masked out.
SSSP_DELTAS = (64, 256, 1024, 4096, 16384, 65536)
SSSP_SOURCES = 8
SSSP_NEAR_BEST = 1.03


def sssp_times(ctx, dgraph, cfgs, src: int = 0, deltas=SSSP_DELTAS, reps: int = 2) -> np.ndarray:
    """t[k, j]: fastest of `reps` SSSP kernel times (ms) under launch
    configuration k and bucket width deltas[j]."""
    g = _g()
    out = ctx.array(dgraph.n, np.int32)
    t = np.full((len(cfgs), len(deltas)), np.inf)
    for k, c in enumerate(cfgs):
        for j, d in enumerate(deltas):
            for _ in range(reps):
                rc, st = dgraph.sssp(src, out, int(d), c)
                g.check(rc, "sssp (policy labels)")
                t[k, j] = min(t[k, j], float(st.kernel_ms))
    out.free()
    return t


def sssp_labels(t: np.ndarray, mean_w: float, deltas=SSSP_DELTAS):
    """(head 2 label, head 3 label) from a time table: the launch label is the
    log-ratio of the two configurations' best times; the width label the mean
    log2(width / mean weight) of the widths within 3 % of the best under the
    faster configuration (the time is flat over a range of widths)."""
    best_k = t.min(axis=1)
    k = int(np.argmin(best_k))
    near = [j for j in range(t.shape[1]) if t[k, j] <= SSSP_NEAR_BEST * best_k[k]]
    y2 = float(np.mean([np.log2(deltas[j] / max(mean_w, 1.0)) for j in near]))
    y3 = float(np.clip(np.log2(max(best_k[0], 1e-6) / max(best_k[1], 1e-6)), -4.0, 4.0))
    return y2, y3


def sssp_collect(ctx, dgraph, cfgs=None, src: int = 0, reps: int = 2):
    """Training rows of one graph: the SSSP features of SSSP_SOURCES sources
    (src and a seeded sample), all with the graph's labels."""
    cfgs = cfgs or launch_candidates()
    t = sssp_times(ctx, dgraph, cfgs, src, reps=reps)
    f0 = dgraph.sssp_features(src)
    mean_w = float(2.0 ** f0[5] - 1.0)
    y2, y3 = sssp_labels(t, mean_w)
    rng = np.random.default_rng(int(dgraph.n) * 7919 + int(dgraph.m))
    srcs = [src] + [int(x) for x in rng.integers(0, dgraph.n, SSSP_SOURCES - 1)]
    X = np.stack([dgraph.sssp_features(s) for s in srcs]).astype(np.float32)
    Y = np.zeros((len(srcs), 4), np.float32)
    M = np.zeros((len(srcs), 4), np.float32)
    Y[:, 2], Y[:, 3] = y2, y3
    M[:, 2], M[:, 3] = 1.0, LAUNCH_WEIGHT / 4.0
    return X, Y, M, {"times_ms": t, "mean_w": mean_w, "y2": y2, "y3": y3}


def sssp_train(ctx, X, Y, M, steps: int = 3000, lr: float = 3e-3, seed: int = 2023):
    """Adam on the GPU (gsrb_mlp_train); returns (params, loss history)."""
    g = _g()
    return g.mlp_train(ctx, g.mlp_init(seed), X, Y, M, steps=steps, lr=lr)
