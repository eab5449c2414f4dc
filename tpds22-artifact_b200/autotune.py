"""Autotuner: picks barrier variant, cluster size, fan-in, wake-up lines, CTAs
per SM, threads and tile size per workload by measuring candidates on the
device, and caches the winners in a JSON file (tuned.json next to this file by
default).

Families (the same split as gsrb_max_coresident):
  barrier   -- the grid-barrier microbenchmark at a fixed CTAs/SM
  reduce    -- gsrb_reduce_i32 on a given device array
  scan      -- gsrb_scan_u32 on a given device array
  bfs       -- gsrb_bfs on a given device graph
Every candidate is timed with CUDA events on the context stream (median of
`reps` launches after one warm-up); candidates the device cannot co-schedule
are skipped (the library refuses them).
"""
from __future__ import annotations

import json
import pathlib
import statistics
import sys

import numpy as np

CACHE = pathlib.Path(__file__).resolve().parent / "tuned.json"


def _g():
    return sys.modules["gsrb_b200"]


def barrier_candidates(k: int):
    g = _g()
    c = [dict(variant=g.BAR_CCG), dict(variant=g.BAR_FLAT), dict(variant=g.BAR_FLIP, fanin_groups=1),
         dict(variant=g.BAR_LOCKFREE)]
    for R in (2, 4, 8):
        for s in (0, 64):
            c.append(dict(variant=g.BAR_FANOUT, wake_lines=R, spin_ns=s))
    for G in (8, 16, 37, 74):
        for R in (4, 8):
            c.append(dict(variant=g.BAR_HIER, fanin_groups=G, wake_lines=R))
    for cl in (2, 4, 8):
        c.append(dict(variant=g.BAR_CLUSTER_FANOUT, cluster=cl, wake_lines=8))
        c.append(dict(variant=g.BAR_CLUSTER, cluster=cl, fanin_groups=1))
    return c


def _median_ms(ctx, fn, reps):
    ts = []
    for i in range(reps + 1):
        ctx.record(40)
        st = fn()
        if st:
            return None
        ctx.record(41)
        t = ctx.elapsed_ms(40, 41)
        if i:
            ts.append(t)
    if ctx.status()[0] != 0:
        return None
    return statistics.median(ts)


def tune_barrier(ctx, k: int, threads: int = 256, episodes: int = 4000, reps: int = 3, fma: int = 0):
    """Best barrier configuration for k CTAs per SM with `fma` dependent FMAs per
    thread before each episode; returns (cfg dict, ns/episode, table)."""
    g = _g()
    grid = k * ctx.num_sms
    sink = ctx.array(grid * threads, np.float32).zero()
    cnt = ctx.array(1, np.uint32).zero()
    base = _median_ms(ctx, lambda: ctx.barrier_bench(g.cfg(variant=g.BAR_NONE, ctas_per_sm=k, threads=threads),
                                                     episodes, fma, sink, cnt), reps)
    table = []
    for cand in barrier_candidates(k):
        c = g.cfg(ctas_per_sm=k, threads=threads, **cand)
        t = _median_ms(ctx, lambda: ctx.barrier_bench(c, episodes, fma, sink, cnt), reps)
        if t is not None and base is not None:
            table.append((round((t - base) * 1e6 / episodes, 1), cand))
    table.sort(key=lambda x: x[0])
    best = dict(table[0][1], ctas_per_sm=k, threads=threads)
    return best, table[0][0], table


def tune_scan(ctx, d_in, d_out, n: int, reps: int = 3):
    """FANOUT and HIER run the warp-specialised scan (readers one segment ahead
    of writers); FLIP and CCG the single-role pipelined one."""
    g = _g()
    table = []
    for chunk in (32768, 49152, 65536):
        for k, threads in ((1, 1024), (2, 512)):
            for cand in (dict(variant=g.BAR_FANOUT, wake_lines=4), dict(variant=g.BAR_HIER, fanin_groups=16, wake_lines=8),
                         dict(variant=g.BAR_FLIP, fanin_groups=1), dict(variant=g.BAR_CCG)):
                c = g.cfg(ctas_per_sm=k, threads=threads, tile=chunk, **cand)
                t = _median_ms(ctx, lambda: ctx.scan(d_in, d_out, n, c), reps)
                if t is not None:
                    table.append((t, dict(cand, ctas_per_sm=k, threads=threads, tile=chunk)))
    table.sort(key=lambda x: x[0])
    return table[0][1], table[0][0], table


def reduce_stream_ms(ctx, bufs, n: int, out, c, passes: int = 4):
    """Per-launch time (ms) of gsrb_reduce_i32 run back to back over the input
    buffers in turn (launch i reads bufs[i % len(bufs)] and writes
    out[i % len(bufs)]).  The buffers together are larger than L2, so every
    launch reads its input from HBM.  The launches are captured once in a CUDA
    graph and the replay is timed, so the host's call overhead is not in the
    measured time (each launch's own device-side start-up still is).  One
    untimed call per buffer first (it also warms the library's caches, so that
    nothing but the launches is captured)."""
    g = _g()
    nb = len(bufs)
    for i in range(nb):
        if ctx.reduce_i32(bufs[i], n, out.at(i), c):
            return None
    if ctx.status()[0] != 0:
        return None
    cg = g.CudaGraph(ctx)
    with cg:
        for i in range(passes * nb):
            g.check(ctx.reduce_i32(bufs[i % nb], n, out.at(i % nb), c), "reduce (capture)")
    try:
        cg.launch()  # untimed replay
        ctx.record(40)
        cg.launch()
        ctx.record(41)
        t = ctx.elapsed_ms(40, 41)
    finally:
        cg.free()
    if ctx.status()[0] != 0:
        return None
    return t / (passes * nb)


def reduce_candidates(k: int | None = None, threads: int | None = None, overlap: bool = False):
    """The library's own barrier protocols (and grid.sync for comparison) at
    the given shape, or over the shapes the reduce supports.  overlap: also
    the chained form of the plain-launch protocols (cfg.overlap = 1: a launch
    may start streaming its input while the previous reduction on the stream
    finishes; valid when that reduction does not write this one's input)."""
    g = _g()
    shapes = [(k, threads)] if k else [(1, 1024), (1, 512), (2, 512), (2, 256), (4, 256)]
    out = []
    for kk, th in shapes:
        for stages in (0, 2, 1):
            for cand in (dict(variant=g.BAR_FANOUT, wake_lines=4), dict(variant=g.BAR_FLIP, fanin_groups=1),
                         dict(variant=g.BAR_HIER, fanin_groups=16, wake_lines=4), dict(variant=g.BAR_CCG)):
                out.append(dict(cand, ctas_per_sm=kk, threads=th, tile=stages))
                if overlap and cand["variant"] != g.BAR_CCG:
                    out.append(dict(cand, ctas_per_sm=kk, threads=th, tile=stages, overlap=1))
    return out


def tune_reduce(ctx, bufs, n: int, out, k: int | None = None, threads: int | None = None, passes: int = 3,
                library_barrier_only: bool = True, overlap: bool = False):
    """Fastest configuration by reduce_stream_ms; with library_barrier_only the
    cooperative-groups barrier is timed but not chosen; overlap: the chained
    form is a candidate too."""
    g = _g()
    table = []
    for e in reduce_candidates(k, threads, overlap):
        t = reduce_stream_ms(ctx, bufs, n, out, g.cfg(**e), passes)
        if t is not None:
            table.append((t, e))
    table.sort(key=lambda x: x[0])
    pick = [r for r in table if not (library_barrier_only and r[1]["variant"] == g.BAR_CCG)]
    return pick[0][1], pick[0][0], table


def segment_candidates(kind: str):
    """Shapes and sub-grid protocols for the batched segment calls (protocols
    whose state does not depend on the team size; for the scan also the round
    length: 1, 2, 4 (= 0, the default) or 8 tiles of 16 x threads per CTA -- a
    short round keeps the round and its prefetched successor in L2 for the
    rescan, a long one pays fewer barriers), and the register-resident form
    that keeps each round's chunk in registers."""
    g = _g()
    out = []
    for k, threads in ((2, 512), (4, 256), (8, 128), (2, 256), (1, 1024)):
        for cand in (dict(variant=g.BAR_FANOUT, wake_lines=4), dict(variant=g.BAR_FLIP, fanin_groups=1),
                     dict(variant=g.BAR_FLAT)):
            for tile in ((16 * threads, 2 * 16 * threads, 0, 8 * 16 * threads) if kind == "scan" else (0,)):
                out.append(dict(cand, ctas_per_sm=k, threads=threads, tile=tile))
    if kind == "scan":
        # register-resident rounds (fan-out only): two groups a CTA; the chunk
        # is threads x 4 x (16 vectors a lane when an SM holds <= 512 of the
        # launch's threads, else 8) / 2
        for k, threads in ((4, 256), (2, 512), (4, 128), (2, 256)):
            per = threads * (16 if k * threads <= 512 else 8) * 4
            out.append(dict(variant=g.BAR_FANOUT, wake_lines=4, ctas_per_sm=k, threads=threads, form=g.FORM_REG,
                            tile=per // 2))
    return out


def tune_segments(ctx, kind: str, d_in, d_out, offsets, reps: int = 3):
    """Best configuration of gsrb_reduce_i32_segments (kind "reduce", d_out =
    the sums) or gsrb_scan_u32_segments (kind "scan"), timed cold (L2 flushed)."""
    g = _g()
    table = []
    for cand in segment_candidates(kind):
        c = g.cfg(**cand)

        def run():
            ctx.l2_flush()
            if kind == "reduce":
                return ctx.reduce_i32_segments(d_in, offsets, d_out, c)
            return ctx.scan_u32_segments(d_in, d_out, offsets, c)
        t = _median_ms(ctx, run, reps)
        if t is not None:
            table.append((t, cand))
    table.sort(key=lambda x: x[0])
    return table[0][1], table[0][0], table


def tune_bfs(ctx, dgraph, src: int, mode: int, reps: int = 2, library_barrier_only: bool = True):
    """Fastest launch shape and barrier for a BFS; with library_barrier_only
    the cooperative-groups barrier is timed but not chosen."""
    g = _g()
    out = ctx.array(dgraph.n, np.int32)
    table = []
    # small grids matter on meshes (one SM's worth of CTAs of 256 threads
    # runs the 2048^2 grid's 4095 levels fastest: fewer barrier participants)
    for k, threads in ((1, 512), (2, 256), (2, 512), (4, 256), (1, 256), (1, 128)):
        for cand in (dict(variant=g.BAR_FANOUT, wake_lines=4), dict(variant=g.BAR_FLIP, fanin_groups=1),
                     dict(variant=g.BAR_HIER, fanin_groups=16, wake_lines=8), dict(variant=g.BAR_CCG)):
            c = g.cfg(ctas_per_sm=k, threads=threads, **cand)
            ts = []
            for _ in range(reps):
                rc, st = dgraph.bfs(src, out, mode, c)
                if rc:
                    ts = None
                    break
                ts.append(st.kernel_ms)
            if ts:
                table.append((statistics.median(ts), dict(cand, ctas_per_sm=k, threads=threads)))
    table.sort(key=lambda x: x[0])
    pick = [r for r in table if not (library_barrier_only and r[1]["variant"] == g.BAR_CCG)]
    return pick[0][1], pick[0][0], table


def load_cache(path=CACHE) -> dict:
    try:
        return json.loads(pathlib.Path(path).read_text())
    except Exception:
        return {}


def save_cache(data: dict, path=CACHE):
    pathlib.Path(path).write_text(json.dumps(data, indent=1, sort_keys=True))


def cfg_from(entry: dict):
    g = _g()
    keys = {k: v for k, v in entry.items() if k in dict(g.Cfg._fields_)}
    return g.cfg(**keys)
