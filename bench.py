#!/usr/bin/env python
"""Benchmark driver: one JSON line on rank 0.

Headline workload (the configuration the metric's first clause is quoted on):
the grid-barrier microbenchmark -- one persistent launch of 148*k CTAs x 256
threads running 10,000 barrier episodes, k = 8 (full residency: 2048 threads
per SM), each episode preceded by F = 0 dependent FP32 FMAs per thread.
value = ns per grid barrier = (t_launch - t_phase_only) / episodes (lower is
better), with the barrier configuration chosen by the autotuner at run time.

The same line carries every other configuration of the benchmark plan,
measured on the same device in the same run (disable with --no-extras):
  barrier_table     ns/episode for k in {1,2,4,8} x F in {0,64,1024}: tuned
                    native barrier vs cooperative-groups grid.sync and the
                    reference algorithms (GSRB, GCPUSRB, atomic tree, lock-free tree)
  semaphore         acquires/s, capacity S in {1,2,10,120}, 1 writer per 10 readers
  reduce_2e24       GB/s and fraction of measured HBM (cold L2), bit-exact check
  scan_2e28         u32 (bit-exact) and f32 (1e-5 relative), GB/s, HBM fraction
  graphs            RMAT-22 and the 2048^2 grid: BFS (plain push / heuristic /
                    learned), SSSP, PageRank; GTEPS; levels/distances checked
  batch             64 RMAT graphs (scales 14..20): plain one-by-one push BFS vs
                    batched + learned in one CUDA-graph launch; aggregate GTEPS

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload barrier|reduce|scan|bfs|sssp|pr|prr] [--graph rmat|grid] [--scale 22]
                  [--k 8] [--fma 0] [--cfg JSON] [--no-extras]

--impl reference times the reference's CPU implementation of the path on the
host cores: the reference has no CPU barrier, so this is the oracle's port of
its sense-reversing barrier run by host threads (same metric and unit).
Multi-GPU: the barrier does not shard (replicas only): every rank runs the
same workload on its own GPU and the reported time is the max over ranks; the
other configurations are measured at N = 1 only.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import pathlib
import re
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
PKG = ROOT / "tpds22-artifact_b200"
PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
SEED = 0x5EED2022


def _load(name, path):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_binding():
    return _load("gsrb_b200", PKG / "gsrb.py")


def load_oracle():
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_binding  # the checker / CPU-baseline leg only
    return oracle_binding


def hbm_peak():
    try:
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


def wall(fn):
    """(seconds, result) of one call: the CPU-baseline leg's clock."""
    t0 = time.perf_counter()
    r = fn()
    return time.perf_counter() - t0, r


def cpu_info():
    """Host CPU model and logical core count (recorded with every CPU baseline)."""
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count() or 1}


# ---------------------------------------------------------------- distributed
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for name, val in zip(names, r[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------- barrier
def time_barrier(gsrb, ctx, c, episodes, fma, steps, warmup, flush=True):
    """Per-launch CUDA-event times (ms) of `steps` launches after `warmup`."""
    grid = c.ctas_per_sm * ctx.num_sms if c.grid_override <= 0 else c.grid_override
    sink = ctx.array(grid * c.threads, np.float32).zero()
    cnt = ctx.array(1, np.uint32).zero()
    times = []
    for i in range(warmup + steps):
        if flush:
            ctx.l2_flush()
        ctx.record(0)
        gsrb.check(ctx.barrier_bench(c, episodes, fma, sink, cnt), "barrier_bench")
        ctx.record(1)
        ms = ctx.elapsed_ms(0, 1)
        if i >= warmup:
            times.append(ms)
    ctx.check_status("barrier_bench")
    total = int(cnt.download()[0])
    assert total == (warmup + steps) * episodes * grid, f"episode count {total}"
    sink.free()
    cnt.free()
    return times


def barrier_e2e(gsrb, ctx, c, episodes, fma, steps, warmup):
    """The same launch through the public C ABI with host buffers: H2D of the
    per-thread FMA seeds from pinned memory, the launch, D2H of the results."""
    import ctypes as C
    lib = gsrb.lib()
    grid = c.ctas_per_sm * ctx.num_sms
    n = grid * c.threads
    h_in, h_out = C.c_void_p(), C.c_void_p()
    gsrb.check(lib.gsrb_host_alloc(C.byref(h_in), n * 4))
    gsrb.check(lib.gsrb_host_alloc(C.byref(h_out), n * 4 + 4))
    C.memset(h_in, 0, n * 4)
    sink = ctx.array(n, np.float32)
    cnt = ctx.array(1, np.uint32).zero()
    times = []
    for i in range(warmup + steps):
        ctx.l2_flush()
        ctx.record(2)
        gsrb.check(lib.gsrb_memcpy_h2d(ctx.h, sink.ptr, h_in, n * 4))
        gsrb.check(ctx.barrier_bench(c, episodes, fma, sink, cnt))
        gsrb.check(lib.gsrb_memcpy_d2h(ctx.h, h_out, sink.ptr, n * 4))
        gsrb.check(lib.gsrb_memcpy_d2h(ctx.h, h_out.value + n * 4, cnt.ptr, 4))
        ctx.record(3)
        ms = ctx.elapsed_ms(2, 3)
        if i >= warmup:
            times.append(ms)
    ctx.check_status("e2e")
    lib.gsrb_host_free(h_in)
    lib.gsrb_host_free(h_out)
    return times, n * 4, n * 4 + 4


def l2_atomic_peak(ctx):
    """Same-address red.add throughput (atomics/s) and atom round trip (ns)."""
    ctas, iters = 4 * ctx.num_sms, 2000
    ctx.probe_l2_atomics(ctas, 200, 0)
    ms = min(ctx.probe_l2_atomics(ctas, iters, 0) for _ in range(3))
    rate = ctas * iters / (ms * 1e-3)
    # the round trip is one CTA's dependent chain: the fastest of several runs
    # after a longer warm-up (a single slow sample once doubled it)
    ctx.probe_l2_atomics(1, 5000, 1)
    ms1 = min(ctx.probe_l2_atomics(1, 20000, 1) for _ in range(7))
    return rate, ms1 * 1e6 / 20000


def arrivals_per_episode(gsrb, c, grid):
    if c.variant in (gsrb.BAR_CLUSTER, gsrb.BAR_CLUSTER_ALLPOLL, gsrb.BAR_DSMEM, gsrb.BAR_CLUSTER_RED,
                     gsrb.BAR_CLUSTER_FANOUT):
        return grid // max(1, c.cluster)
    return grid


def barrier_table(gsrb, ctx, tune, tuned_cache):
    """ns/episode for k in {1,2,4,8} x F in {0,64,1024}: the barrier tuned for
    that (k, F) against cooperative groups and the reference algorithms."""
    rows = []
    for k in (1, 2, 4, 8):
        for F in (0, 64, 1024):
            eps = 2000 if F < 1024 else 500
            best, _, _ = tune.tune_barrier(ctx, k, episodes=eps, reps=2, fma=F)
            tuned_cache[f"barrier_k{k}_F{F}"] = best
            bc = tune.cfg_from(best)
            base = statistics.median(time_barrier(gsrb, ctx, gsrb.cfg(variant=gsrb.BAR_NONE, ctas_per_sm=k,
                                                                     threads=256), eps, F, 3, 1))
            row = {"k": k, "F": F, "tuned": gsrb.VARIANT_NAMES[best["variant"]]}
            for name, c in (("native", bc), ("ccg", gsrb.cfg(variant=gsrb.BAR_CCG, ctas_per_sm=k, threads=256)),
                            ("ref_gsrb", gsrb.cfg(variant=gsrb.BAR_SOFT2, ctas_per_sm=k, threads=256)),
                            ("ref_gcpusrb", gsrb.cfg(variant=gsrb.BAR_FLAT, ctas_per_sm=k, threads=256)),
                            ("atomic_tree", gsrb.cfg(variant=gsrb.BAR_TREE, ctas_per_sm=k, threads=256)),
                            ("ref_lockfree", gsrb.cfg(variant=gsrb.BAR_LOCKFREE, ctas_per_sm=k, threads=256))):
                try:
                    t = statistics.median(time_barrier(gsrb, ctx, c, eps, F, 3, 1))
                    row[name] = round((t - base) * 1e6 / eps, 1)
                except (gsrb.GsrbError, AssertionError) as e:
                    row[name] = f"failed: {e}"
            if isinstance(row.get("ccg"), float) and isinstance(row.get("native"), float):
                row["speedup_vs_ccg"] = round(row["ccg"] / max(row["native"], 1e-9), 3)
            rows.append(row)
    return rows


def semaphore_numbers(gsrb, ctx):
    """Acquires/s of the priority semaphore (148 x 8 CTAs, one writer per 10
    readers, 100 increments per hold, 2 holds per CTA) beside the reference's
    protocols restated.  For scale, the holds' own cost: with one CTA and no
    semaphore (GSRB_SEM_NONE) a writer's hold takes T_w and a reader's T_r, and
    "serial_holds_acq_per_s" is the rate of W writer holds back to back plus R
    reader holds S at a time at those costs.  It is not a bound: one CTA's
    holds pay its own SM's distance to the counters' L2 slice, while the
    contended run spreads writers over both dies."""
    iters, incs, every, k = 2, 100, 11, 8

    def bare(writer_every, r1=100, r2=1100):
        # the call's own set-up (lock state allocation, record init) is in both
        # timings: the difference over r2 - r1 holds is the holds alone
        c = gsrb.cfg(ctas_per_sm=1, threads=256, grid_override=1)
        cnt = ctx.array(8, np.uint32).zero()
        ts = []
        for reps in (r1, r2, r1, r2):
            cnt.zero()
            ctx.record(6)
            gsrb.check(ctx.semaphore_bench(c, gsrb.SEM_NONE, 1, writer_every, reps, incs, cnt), "semaphore probe")
            ctx.record(7)
            ts.append(ctx.elapsed_ms(6, 7))
        return max(1e-6, (min(ts[1], ts[3]) - min(ts[0], ts[2])) / (r2 - r1))

    t_w, t_r = bare(1), bare(0)
    grid = k * ctx.num_sms
    writers = len([b for b in range(grid) if b % every == 0])
    out = []
    for S in (1, 2, 10, 120):
        bound_ms = writers * iters * t_w + (grid - writers) * iters * t_r / S
        rate_bound = grid * iters / (bound_ms * 1e-3)
        row = {"S": S, "serial_holds_acq_per_s": round(rate_bound, 1)}
        for name, kind in (("native_priority", gsrb.SEM_PRIORITY), ("ref_priority", gsrb.SEM_REF_PRIORITY),
                           ("ref_spin", gsrb.SEM_REF_SPIN)):
            c = gsrb.cfg(ctas_per_sm=k, threads=256, timeout_ms=5000)
            cnt = ctx.array(8, np.uint32).zero()
            ctx.record(6)
            st = ctx.semaphore_bench(c, kind, S, every, iters, incs, cnt)
            ctx.record(7)
            ms = ctx.elapsed_ms(6, 7)
            W, R, inside, maxr, viol, acq, tmo, _ = cnt.download().tolist()
            exact = (st == 0 and W == writers * iters * incs and R == (grid - writers) * iters * incs and viol == 0
                     and maxr <= S)
            rate = acq / (ms * 1e-3)
            row[name] = {"acquires_per_s": round(rate, 1), "ms": round(ms, 3), "exact": exact, "ctas": grid,
                         "x_serial_holds": round(rate / rate_bound, 4)}
        out.append(row)
    return {"rows": out, "writer_hold_us": round(t_w * 1e3, 3), "reader_hold_us": round(t_r * 1e3, 3),
            "shape": f"{grid} CTAs x 256 threads, 1 writer per {every - 1} readers, {incs} increments per hold, "
                     f"{iters} holds per CTA"}


# --------------------------------------------------------------- data kernels
def reduce_numbers(gsrb, ctx, orc, tune, cache, reps=10, fixed=None, n=1 << 24, cpu=False):
    """The C1 reduce: 2^24 int32 U[0,127], grid 148 x 2 CTAs x 256 threads.
    Timed as a stream of reductions: launches back to back over several
    inputs that together exceed four times the L2 (each launch reads its input
    from HBM); value = per-launch time.  Chained launches (cfg.overlap: a
    launch starts streaming its input while the previous one combines) are
    candidates, and the best unchained configuration is reported beside.  The configuration is the fastest of the
    library's own barrier protocols at the C1 shape (grid.sync is timed beside
    it); the fastest over every shape is reported too, and so is one launch
    alone after an L2 flush (the launch overhead included)."""
    # at least four L2 sizes of inputs, read round robin: an input's lines are
    # gone from L2 by the time it comes round again
    nb = int(min(64, max(2, -(-4 * ctx.l2_bytes // (4 * n)))))
    inputs = [gsrb.uniform_i32(SEED + i, n, 0, 127) for i in range(nb)]
    bufs = [ctx.to_device(a) for a in inputs]
    out = ctx.array(nb, np.int64).zero()
    if fixed:
        best, table = fixed, []
    else:
        # chained launches (cfg.overlap) are valid here: the inputs are all
        # ready before the stream begins and no reduction writes another's input
        best, _, table = tune.tune_reduce(ctx, bufs, n, out, k=2, threads=256, overlap=True)
    cache["reduce"] = best
    c = tune.cfg_from(best)
    times = [tune.reduce_stream_ms(ctx, bufs, n, out, c, passes=max(1, reps // 2)) for _ in range(3)]
    ctx.check_status("reduce")
    got = out.download()
    ok = all(int(got[i]) == orc.sum_i32(inputs[i]) for i in range(nb))
    t = statistics.median(times)
    peak, src = hbm_peak()
    gbs = 4 * n / (t * 1e-3) / 1e9
    res = {"n": n, "ms": round(t, 5), "GB_s": round(gbs, 1), "hbm_frac": round(gbs / peak, 4),
           "peak_source": src, "bit_exact": ok, "cfg": best,
           "timing": f"{nb} inputs of {4 * n} B ({4 * n * nb} B in all, > 4x L2) reduced in turn, back to back, "
                     "the launches replayed from a CUDA graph; per-launch time"}
    ccg = [r for r in table if r[1]["variant"] == gsrb.BAR_CCG]
    if ccg:
        res["ccg_ms"] = round(min(r[0] for r in ccg), 5)
    unchained = [r for r in table if r[1]["variant"] != gsrb.BAR_CCG and not r[1].get("overlap")]
    if unchained:
        tu, cu = min(unchained, key=lambda r: r[0])
        res["unchained"] = {"ms": round(tu, 5), "hbm_frac": round(4 * n / (tu * 1e-3) / 1e9 / peak, 4), "cfg": cu,
                            "note": "each launch waits for the previous one to finish (no programmatic "
                                    "dependent launch)"}
    if not fixed:
        anyb, tany, _ = tune.tune_reduce(ctx, bufs, n, out)
        res["tuned_any_shape"] = {"ms": round(tany, 5), "hbm_frac": round(4 * n / (tany * 1e-3) / 1e9 / peak, 4),
                                  "cfg": anyb}
    # one launch alone, L2 flushed before it (launch latency and ramp included)
    single = []
    # the best unchained configuration (a chained launch's shape is picked for overlap)
    c1 = tune.cfg_from(min(unchained, key=lambda r: r[0])[1] if unchained else dict(best, overlap=0))
    for i in range(8):
        ctx.l2_flush()
        ctx.record(4)
        gsrb.check(ctx.reduce_i32(bufs[0], n, out.at(0), c1))
        ctx.record(5)
        if i >= 3:
            single.append(ctx.elapsed_ms(4, 5))
    res["single_launch_cold_us"] = round(statistics.median(single) * 1e3, 2)
    for bb in bufs:
        bb.free()
    a = inputs[0]
    if cpu:
        thr = os.cpu_count() or 1
        t1 = statistics.median(wall(lambda: orc.sum_i32(a))[0] for _ in range(5))
        tm = statistics.median(wall(lambda: orc.sum_i32(a, threads=thr))[0] for _ in range(5))
        res["cpu"] = {"kind": "port", "serial_ms": round(t1 * 1e3, 3), "serial_GB_s": round(4 * n / t1 / 1e9, 2),
                      "mt_ms": round(tm * 1e3, 3), "mt_GB_s": round(4 * n / tm / 1e9, 2), "threads": thr,
                      "sample": f"the same {n} int32, int64 sum, median of 5", **cpu_info()}
    return res


def scan_numbers(gsrb, ctx, orc, tune, cache, n=1 << 28, reps=5, fixed=None, cpu=False):
    peak, src = hbm_peak()
    res = {"n": n, "peak_source": src}
    a = gsrb.uniform_i32(SEED, n, 0, 15).astype(np.uint32)
    din = ctx.to_device(a)
    dout = ctx.array(n, np.uint32)
    best = fixed or tune.tune_scan(ctx, din, dout, n, reps=2)[0]
    cache["scan"] = best
    c = tune.cfg_from(best)
    for kind in ("u32", "f32"):
        if kind == "f32":
            din.free()
            dout.free()
            a = gsrb.uniform_f32(SEED, n)
            din = ctx.to_device(a)
            dout = ctx.array(n, np.float32)
        times = []
        for i in range(1 + reps):
            ctx.record(4)
            gsrb.check(ctx.scan(din, dout, n, c))
            ctx.record(5)
            if i:
                times.append(ctx.elapsed_ms(4, 5))
        ctx.check_status("scan")
        got = dout.download()
        if kind == "u32":
            thr = os.cpu_count() or 1
            t_mt, want = wall(lambda: orc.scan_u32(a, threads=thr))
            ok = bool(np.array_equal(got, want))
            check = {"bit_exact": ok}
            if cpu:
                t_ref, ref_out = wall(lambda: orc.ref_cpu_sum_scan(a))
                res["cpu"] = {"kind": "reference" if ref_out is not None else "port",
                              "serial_ms": round(t_ref * 1e3, 1) if ref_out is not None else None,
                              "serial_GB_s": round(8 * n / t_ref / 1e9, 2) if ref_out is not None else None,
                              "serial_matches": bool(np.array_equal(ref_out, want)) if ref_out is not None else None,
                              "mt_ms": round(t_mt * 1e3, 1), "mt_GB_s": round(8 * n / t_mt / 1e9, 2), "threads": thr,
                              "sample": f"the same {n} uint32: the reference's cpu_sum_scan (scan/main.cu:11-21, "
                                        f"oracle/_ref) on one core; the two-pass blocked scan on all cores",
                              **cpu_info()}
                del ref_out
            del want
        else:
            ref = orc.scan_f32_f64(a)
            err = orc.max_rel_err(got[1:], ref[1:])
            check = {"max_rel_err": err, "within_1e-5": bool(err <= 1e-5)}
            del ref
        del got
        t = statistics.median(times)
        gbs = 8 * n / (t * 1e-3) / 1e9
        res[kind] = dict({"ms": round(t, 4), "GB_s": round(gbs, 1), "hbm_frac": round(gbs / peak, 4)}, **check)
    res["cfg"] = best
    din.free()
    dout.free()
    return res


# --------------------------------------------------------------------- graphs
def train_policy(gsrb, ctx, pol):
    """Per-level traces of training graphs (not the evaluation graphs) -> MLP."""
    graphs = [gsrb.rmat(s, 16, seed=SEED + 1000 + s) for s in (14, 16, 18, 20, 21, 22)]
    graphs += [gsrb.grid2d(256, 256, seed=SEED + 7), gsrb.grid2d(1024, 64, seed=SEED + 8),
               gsrb.grid2d(1024, 1024, seed=SEED + 9), gsrb.grid2d(2048, 512, seed=SEED + 10),
               gsrb.grid2d(4096, 1024, seed=SEED + 11), gsrb.grid2d(3072, 1536, seed=SEED + 12)]
    X, Y, M = [], [], []
    cands = pol.launch_candidates()
    launch = []
    for g in graphs:
        dg = ctx.graph(g)
        x, y, m, info = pol.collect(ctx, dg, 0, reps=2, launch_cfgs=cands)
        launch.append([g.nnodes, g.nedges] + [round(float(t), 3) for t in info["launch_ms"]])
        X.append(x)
        Y.append(y)
        M.append(m)
        dg.free()
    X, Y, M = np.concatenate(X), np.concatenate(Y), np.concatenate(M)
    t0 = time.time()
    params, hist = pol.train(ctx, X, Y, M, steps=3000)
    acc = pol.accuracy(ctx, params, X, Y, M)
    return params, {"levels": int(len(X)), "train_s": round(time.time() - t0, 2), "loss_first": float(hist[0]),
                    "loss_last": float(hist[-1]), **acc,
                    "launch_labels": {"candidates": [gsrb.VARIANT_NAMES[c.variant] + f" {c.ctas_per_sm}x{c.threads}"
                                                     for c in cands],
                                      "n_m_ms0_ms1": launch}}


def bfs_runs(gsrb, ctx, orc, dg, g, params, cfg, reps=3, launch=None, cpu=False):
    out = ctx.array(g.nnodes, np.int32)
    t_cpu, want = wall(lambda: orc.bfs(g, 0))
    m_trav = orc.traversed_edges(g, want)
    res = {"m_traversed": m_trav}
    if cpu:
        thr = os.cpu_count() or 1
        t_mt, got = wall(lambda: orc.bfs(g, 0, threads=thr))
        res["cpu"] = {"kind": "port", "serial_ms": round(t_cpu * 1e3, 2),
                      "serial_GTEPS": round(m_trav / t_cpu / 1e9, 4), "mt_ms": round(t_mt * 1e3, 2),
                      "mt_GTEPS": round(m_trav / t_mt / 1e9, 4), "mt_matches": bool(np.array_equal(got, want)),
                      "threads": thr, "sample": "one whole BFS from vertex 0: queue BFS on one core, "
                                                "level-synchronous BFS on all cores"}
    dg.set_policy(params)
    for name, mode in (("plain_push", gsrb.BFS_PUSH), ("push_load_balanced", gsrb.BFS_PUSH | gsrb.BFS_FLAG_LB),
                       ("heuristic", gsrb.BFS_HEURISTIC), ("learned", gsrb.BFS_LEARNED)):
        ts = []
        for _ in range(reps):
            rc, st = dg.bfs(0, out, mode, cfg)
            gsrb.check(rc, f"bfs {name}")
            ts.append(st.kernel_ms)
        ok = bool(np.array_equal(out.download(), want))
        t = statistics.median(ts)
        res[name] = {"ms": round(t, 3), "GTEPS": round(m_trav / (t * 1e-3) / 1e9, 3), "levels": int(st.levels),
                     "bit_exact": ok}
        if mode == gsrb.BFS_LEARNED:
            res[name]["policy_decisions"] = int(st.decisions)
            res[name]["fallback_level"] = int(st.aux)
            if st.levels <= 64:
                # per-level schedule (0 push, 1 pull, 2 topology push, 3 one-CTA push)
                res[name]["dirs"] = [int(x) for x in dg.trace(64)["dir"][: int(st.levels)]]
    res["learned_vs_plain"] = round(res["plain_push"]["ms"] / res["learned"]["ms"], 3)
    if launch is not None:
        # the policy's head 3 also picks the launch (barrier variant and CTA
        # shape) between two fixed candidates, with no autotuning; the learned
        # traversal's time under each candidate shows whether it chose well
        each = []
        for c in launch:
            ts = []
            for _ in range(reps):
                rc, st = dg.bfs(0, out, gsrb.BFS_LEARNED, c)
                gsrb.check(rc, "bfs learned (launch candidate)")
                ts.append(st.kernel_ms)
            each.append(round(statistics.median(ts), 3))
        dg.set_launch_choices(*launch)
        ts = []
        for _ in range(reps):
            rc, st = dg.bfs(0, out, gsrb.BFS_LEARNED)
            gsrb.check(rc, "bfs learned (own launch)")
            ts.append(st.kernel_ms)
        ok = bool(np.array_equal(out.download(), want))
        k, z = dg.policy_launch(0)
        dg.set_launch_choices(None, None)
        t = statistics.median(ts)
        res["learned_own_launch"] = {"ms": round(t, 3), "GTEPS": round(m_trav / (t * 1e-3) / 1e9, 3),
                                     "launch": int(st.launch) - 1, "head3": round(z, 3),
                                     "candidates_ms": each,
                                     "candidates": [gsrb.VARIANT_NAMES[c.variant] + f" {c.ctas_per_sm}x{c.threads}"
                                                    for c in launch],
                                     "bit_exact": ok}
    return res


def sssp_runs(gsrb, ctx, orc, dg, g, deltas, cfg, verify=True):
    out = ctx.array(g.nnodes, np.int32)
    t_cpu, want = wall(lambda: orc.dijkstra(g, 0)) if verify else (None, None)
    m_trav = orc.traversed_edges(g, want) if verify else g.nedges
    res = {}
    if verify:
        res["cpu"] = {"kind": "port", "serial_ms": round(t_cpu * 1e3, 2),
                      "serial_GTEPS": round(m_trav / t_cpu / 1e9, 4), "threads": 1,
                      "sample": "one whole binary-heap Dijkstra from vertex 0 on one core"}
    for name, delta, *rest in deltas:
        c = rest[0] if rest else cfg  # an arm may bring its own launch configuration (None: the default
        # one, or the SSSP policy's choice when delta is SSSP_DELTA_LEARNED)
        ts = []
        for _ in range(3):
            rc, st = dg.sssp(0, out, delta, c)
            gsrb.check(rc, "sssp")
            ts.append(st.kernel_ms)
        ms = statistics.median(ts[1:])
        ok = bool(np.array_equal(out.download(), want)) if verify else None
        res[name] = {"delta": int(st.delta), "launch": int(st.launch), "ms": round(ms, 3),
                     "GTEPS": round(m_trav / (ms * 1e-3) / 1e9, 3), "rounds": int(st.levels),
                     "buckets": int(st.aux), "edges_relaxed": int(st.edges), "bit_exact": ok}
    return res


def train_sssp_policy(gsrb, ctx, pol):
    """SSSP policy from timed runs of training graphs (not the evaluated ones):
    every width of policy.SSSP_DELTAS under both launch candidates."""
    graphs = [gsrb.rmat(s, 16, seed=SEED + 2000 + s) for s in (14, 16, 18, 20, 21)]
    # grids up to 2^21 vertices: on meshes the best width grows with the
    # diameter (fewer rounds), so the network must see large ones
    graphs += [gsrb.grid2d(w, h, seed=SEED + 2100 + w + h, wlo=1, whi=1000)
               for w, h in ((256, 256), (1024, 64), (512, 512), (1024, 1024), (2048, 256), (2048, 1024),
                            (4096, 512))]
    X, Y, M, rows = [], [], [], []
    t0 = time.time()
    for g in graphs:
        dg = ctx.graph(g)
        x, y, m, info = pol.sssp_collect(ctx, dg, reps=1)
        rows.append({"n": g.nnodes, "m": g.nedges, "delta_label_log2": round(info["y2"], 3),
                     "launch_label": round(info["y3"], 3)})
        X.append(x)
        Y.append(y)
        M.append(m)
        dg.free()
    X, Y, M = np.concatenate(X), np.concatenate(Y), np.concatenate(M)
    params, hist = pol.sssp_train(ctx, X, Y, M, steps=3000)
    return params, {"graphs": rows, "rows": int(len(X)), "collect_and_train_s": round(time.time() - t0, 1),
                    "loss_first": float(hist[0]), "loss_last": float(hist[-1])}


def _tuning_note(gsrb, best, table):
    """The tuned launch (the library's own barriers only) and, beside it, the
    fastest shape under grid.sync, from the tuner's timing table."""
    ccg = [r for r in table if r[1]["variant"] == gsrb.BAR_CCG]
    own = [r for r in table if r[1]["variant"] != gsrb.BAR_CCG]
    return {"cfg": best, "tuning_ms": round(own[0][0], 3) if own else None,
            "grid_sync_best_ms": round(ccg[0][0], 3) if ccg else None,
            "grid_sync_best_cfg": ccg[0][1] if ccg else None}


def graph_numbers(gsrb, ctx, orc, pol, params, sparams, tune, cache, verify_pr=True, ref_gpu="quick"):
    res = {}
    t0 = time.time()
    rm = gsrb.rmat(22, 16, a=0.57, b=0.19, c=0.19, seed=SEED, wlo=1, whi=255)
    res["rmat22"] = {"n": rm.nnodes, "m": rm.nedges, "max_degree": int(rm.degrees().max()),
                     "gen_s": round(time.time() - t0, 1)}
    dg = ctx.graph(rm)
    best, _, ttab = tune.tune_bfs(ctx, dg, 0, gsrb.BFS_HEURISTIC, reps=1)
    cache["bfs_rmat"] = best
    res["rmat22"]["launch_tuning"] = _tuning_note(gsrb, best, ttab)
    cfg = tune.cfg_from(best)
    res["rmat22"]["bfs"] = bfs_runs(gsrb, ctx, orc, dg, rm, params, cfg, launch=pol.launch_candidates(), cpu=True)
    dg.set_sssp_policy(sparams)
    dg.set_launch_choices(*pol.launch_candidates())
    res["rmat22"]["sssp"] = sssp_runs(gsrb, ctx, orc, dg, rm, [("learned", gsrb.SSSP_DELTA_LEARNED, None),
                                                              ("reference_delta", 10000, None),
                                                              ("reference_delta_tuned_cfg", 10000),
                                                              ("delta_256", 256, None)], cfg)
    out = ctx.array(rm.nnodes, np.float32)
    rc, st = dg.pagerank(out, 0.85, 50, cfg)
    gsrb.check(rc, "pagerank")
    rc, st = dg.pagerank(out, 0.85, 50, cfg)
    gsrb.check(rc, "pagerank")
    per_iter_bytes = 4 * (rm.nnodes + 1) + 4 * rm.nedges + 8 * rm.nnodes
    l1 = orc.normalized_l1(out.download(), orc.pagerank(rm, 0.85, 50)) if verify_pr else None
    thr = os.cpu_count() or 1
    t_pr1 = wall(lambda: orc.pagerank(rm, 0.85, 5))[0] / 5
    t_prm = wall(lambda: orc.pagerank(rm, 0.85, 5, threads=thr))[0] / 5
    pr_cpu = {"kind": "port", "serial_ms_per_iter": round(t_pr1 * 1e3, 2),
              "serial_edges_per_s": round(rm.nedges / t_pr1, 1), "mt_ms_per_iter": round(t_prm * 1e3, 2),
              "mt_edges_per_s": round(rm.nedges / t_prm, 1), "threads": thr,
              "sample": "5 of the 50 FP64 pull iterations, per-iteration time"}
    # the gather floor: one edge-parallel pass with nothing but the x/deg gathers
    floor_l1, floor_l2 = dg.probe_gather(True), dg.probe_gather(False)
    per_iter = st.kernel_ms / 50
    res["rmat22"]["pagerank_gather_floor"] = {
        "pass_ms_l1": round(floor_l1, 4), "pass_ms_l2": round(floor_l2, 4), "iteration_ms": round(per_iter, 4),
        "frac_of_gather_floor": round(floor_l1 / per_iter, 4),
        "floor_hbm_frac": round(per_iter_bytes / (floor_l1 * 1e-3) / 1e9 / hbm_peak()[0], 4),
        "note": "an edge-parallel pass gathering x/deg at every edge (no per-vertex sums): the most a pull "
                "iteration can reach on this graph; frac = floor / iteration time"}
    res["rmat22"]["pagerank"] = {"iters": 50, "ms": round(st.kernel_ms, 3),
                                 "edges_per_s": round(50 * rm.nedges / (st.kernel_ms * 1e-3), 1),
                                 "GB_s_algorithmic": round(50 * per_iter_bytes / (st.kernel_ms * 1e-3) / 1e9, 1),
                                 "hbm_frac": round(50 * per_iter_bytes / (st.kernel_ms * 1e-3) / 1e9 / hbm_peak()[0], 4),
                                 "l1_vs_fp64": l1, "within_1e-6": (l1 <= 1e-6) if l1 is not None else None,
                                 "cpu": pr_cpu}
    # the reference's push-residual algorithm (epsilon 1e-6, run to empty
    # worklist), checked against the pull form run to convergence (200 iterations)
    conv = ctx.array(rm.nnodes, np.float32)
    gsrb.check(dg.pagerank(conv, 0.85, 200, cfg)[0], "pagerank 200")
    outr = ctx.array(rm.nnodes, np.float32)
    gsrb.check(dg.pagerank_residual(outr, 0.85, 1e-6, 2**31 - 1, cfg)[0], "pagerank_residual")
    rc, st = dg.pagerank_residual(outr, 0.85, 1e-6, 2**31 - 1, cfg)
    gsrb.check(rc, "pagerank_residual")
    res["rmat22"]["pagerank_residual"] = {"epsilon": 1e-6, "ms": round(st.kernel_ms, 3), "rounds": int(st.levels),
                                          "pushes": int(st.edges),
                                          "l1_vs_converged_pull": orc.normalized_l1(outr.download(),
                                                                                    conv.download().astype(np.float64))}
    dg.free()
    if ref_gpu != "none":
        res["rmat22"]["reference_gpu"] = lonestar_reference(rm, "rmat22", ref_gpu)
    del rm
    gr = gsrb.grid2d(2048, 2048, seed=SEED, wlo=1, whi=1000)
    dg = ctx.graph(gr)
    best, _, ttab = tune.tune_bfs(ctx, dg, 0, gsrb.BFS_PUSH, reps=1)
    cache["bfs_grid"] = best
    cfg = tune.cfg_from(best)
    res["grid2048"] = {"n": gr.nnodes, "m": gr.nedges, "launch_tuning": _tuning_note(gsrb, best, ttab),
                       "bfs": bfs_runs(gsrb, ctx, orc, dg, gr, params, cfg, reps=2, launch=pol.launch_candidates(),
                                       cpu=True)}
    dg.set_sssp_policy(sparams)
    dg.set_launch_choices(*pol.launch_candidates())
    res["grid2048"]["sssp"] = sssp_runs(gsrb, ctx, orc, dg, gr, [("learned", gsrb.SSSP_DELTA_LEARNED, None),
                                                                ("reference_delta", 10000, None),
                                                                ("reference_delta_tuned_cfg", 10000),
                                                                ("delta_4096", 4096, None)], cfg)
    dg.free()
    if ref_gpu != "none":
        res["grid2048"]["reference_gpu"] = lonestar_reference(gr, "grid2048", ref_gpu)
    return res


class _At:
    """A device address inside an allocation (a segment's start)."""

    def __init__(self, ptr, dtype):
        self.ptr, self.dtype = ptr, dtype


def segment_numbers(gsrb, ctx, orc, tune, cache, k=64, reps=5, fixed=None):
    """k segments of uneven lengths (2^U(10, 22) elements): one batched launch
    against one persistent launch per segment (the reference's form: one array
    per launch), issued from the host and captured into one CUDA graph."""
    rng = np.random.default_rng(SEED + 64)
    lens = np.round(2.0 ** rng.uniform(10, 22, k)).astype(np.uint64)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    n = int(off[-1])
    peak, src = hbm_peak()
    res = {"segments": k, "elements": n, "min_len": int(lens.min()), "max_len": int(lens.max()),
           "peak_source": src, "cold_l2": True}
    a = gsrb.uniform_i32(SEED + 1, n, 0, 127)
    u = gsrb.uniform_i32(SEED + 2, n, 0, 15).astype(np.uint32)
    da, du = ctx.to_device(a), ctx.to_device(u)
    dsum = ctx.array(k, np.int64).zero()
    dscan = ctx.array(n, np.uint32)
    tune_cfg = gsrb.cfg(**{kk: v for kk, v in cache.get("reduce", {}).items() if kk in dict(gsrb.Cfg._fields_)})
    cs = gsrb.cfg(**{kk: v for kk, v in cache.get("scan", {}).items() if kk in dict(gsrb.Cfg._fields_)})

    def per_segment(kind):
        for i in range(k):
            s0, ln = int(off[i]), int(lens[i])
            if kind == "reduce":
                gsrb.check(ctx.reduce_i32(_At(da.ptr + 4 * s0, np.int32), ln, _At(dsum.ptr + 8 * i, np.int64),
                                          tune_cfg))
            else:
                gsrb.check(ctx.scan(_At(du.ptr + 4 * s0, np.uint32), _At(dscan.ptr + 4 * s0, np.uint32), ln, cs))

    # the batched calls' configurations: fixed, or picked by the autotuner
    cb = {}
    for kind, (din, dout) in (("reduce", (da, dsum)), ("scan", (du, dscan))):
        best = fixed if fixed else tune.tune_segments(ctx, kind, din, dout, off)[0]
        cache["segments_" + kind] = best
        cb[kind] = gsrb.cfg(**{kk: v for kk, v in best.items() if kk in dict(gsrb.Cfg._fields_)})
        res.setdefault("cfg", {})[kind] = best

    def batched(kind):
        if kind == "reduce":
            gsrb.check(ctx.reduce_i32_segments(da, off, dsum, cb[kind]))
        else:
            gsrb.check(ctx.scan_u32_segments(du, dscan, off, cb[kind]))

    def timed(fn):
        ts = []
        for i in range(2 + reps):
            ctx.l2_flush()
            ctx.record(4)
            fn()
            ctx.record(5)
            if i >= 2:
                ts.append(ctx.elapsed_ms(4, 5))
        ctx.check_status("segments")
        return statistics.median(ts)

    want_sum = [orc.sum_i32(a[int(off[i]):int(off[i + 1])]) for i in range(k)]
    want_scan = np.concatenate([orc.scan_u32(u[int(off[i]):int(off[i + 1])]) for i in range(k)])
    for kind, nbytes in (("reduce", 4 * n), ("scan", 8 * n)):
        check = (lambda: dsum.download().tolist() == want_sum) if kind == "reduce" else \
            (lambda: bool(np.array_equal(dscan.download(), want_scan)))
        tb = timed(lambda: batched(kind))
        ok_b = check()
        ts = timed(lambda: per_segment(kind))
        ok_s = check()
        cg = gsrb.CudaGraph(ctx)
        with cg:
            per_segment(kind)
        tg = timed(cg.launch)
        cg.free()
        res[kind] = {"batched_ms": round(tb, 4), "batched_GB_s": round(nbytes / (tb * 1e-3) / 1e9, 1),
                     "batched_hbm_frac": round(nbytes / (tb * 1e-3) / 1e9 / peak, 4),
                     "per_segment_ms": round(ts, 4), "per_segment_graph_ms": round(tg, 4),
                     "speedup_vs_per_segment_graph": round(tg / tb, 3), "bit_exact": bool(ok_b and ok_s)}
    # FP32 segments with the scan's configuration, within 1e-5 relative per element
    f = gsrb.uniform_f32(SEED + 3, n)
    df, dfo = ctx.to_device(f), ctx.array(n, np.float32)
    tf = timed(lambda: gsrb.check(ctx.scan_segments(df, dfo, off, cb["scan"])))
    got = dfo.download()
    err = max((orc.max_rel_err(got[int(off[i]) + 1:int(off[i + 1])],
                               orc.scan_f32_f64(f[int(off[i]):int(off[i + 1])])[1:])
               for i in range(k) if off[i + 1] > off[i] + 1), default=0.0)
    res["scan_f32"] = {"batched_ms": round(tf, 4), "batched_GB_s": round(8 * n / (tf * 1e-3) / 1e9, 1),
                       "batched_hbm_frac": round(8 * n / (tf * 1e-3) / 1e9 / peak, 4),
                       "max_rel_err": err, "within_1e-5": bool(err <= 1e-5)}
    for x in (da, du, dsum, dscan, df, dfo):
        x.free()
    return res


def batch_numbers(gsrb, ctx, orc, params, sparams=None):
    rng = np.random.default_rng(SEED)
    scales = rng.integers(14, 21, 64)
    t0 = time.time()
    graphs = [gsrb.rmat(int(s), 16, seed=SEED + i, wlo=1, whi=255) for i, s in enumerate(scales)]
    gen_s = time.time() - t0
    dgs = [ctx.graph(g) for g in graphs]
    for dg in dgs:
        dg.set_policy(params)
    outs = [ctx.array(g.nnodes, np.int32) for g in graphs]
    t_cpu_bfs, wants = wall(lambda: [orc.bfs(g, 0) for g in graphs])
    m_total = sum(orc.traversed_edges(g, w) for g, w in zip(graphs, wants))
    thr = os.cpu_count() or 1
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(thr) as ex:  # the oracle's C code runs without the GIL
        t_mt_bfs, got = wall(lambda: list(ex.map(lambda g: orc.bfs(g, 0), graphs)))
        mt_ok = all(np.array_equal(a, b) for a, b in zip(got, wants))
        t_cpu_dij, wants_d = wall(lambda: [orc.dijkstra(g, 0) for g in graphs])
        t_mt_dij, got = wall(lambda: list(ex.map(lambda g: orc.dijkstra(g, 0), graphs)))
        mt_ok = mt_ok and all(np.array_equal(a, b) for a, b in zip(got, wants_d))
    del got
    res = {"graphs": 64, "scales": [int(s) for s in scales], "m_total": int(sum(g.nedges for g in graphs)),
           "m_traversed": int(m_total), "gen_s": round(gen_s, 1)}
    res["cpu"] = {"kind": "port", "bfs_serial_ms": round(t_cpu_bfs * 1e3, 1),
                  "bfs_serial_GTEPS": round(m_total / t_cpu_bfs / 1e9, 4),
                  "bfs_mt_ms": round(t_mt_bfs * 1e3, 1), "bfs_mt_GTEPS": round(m_total / t_mt_bfs / 1e9, 4),
                  "sssp_serial_ms": round(t_cpu_dij * 1e3, 1),
                  "sssp_serial_GTEPS": round(m_total / t_cpu_dij / 1e9, 4),
                  "sssp_mt_ms": round(t_mt_dij * 1e3, 1), "sssp_mt_GTEPS": round(m_total / t_mt_dij / 1e9, 4),
                  "mt_matches": mt_ok, "threads": thr,
                  "sample": "all 64 graphs from vertex 0: queue BFS / binary-heap Dijkstra, one graph after "
                            "another on one core, and one graph per host thread on all cores"}
    # plain: the reference algorithm (worklist push), one whole-grid launch per graph
    plain_cfg = gsrb.cfg(variant=gsrb.BAR_SOFT2, ctas_per_sm=2, threads=256)
    for rep in range(2):
        ctx.record(8)
        for dg, o in zip(dgs, outs):
            rc, _ = dg.bfs(0, o, gsrb.BFS_PUSH, plain_cfg)
            gsrb.check(rc, "plain bfs")
        ctx.record(9)
        t_plain = ctx.elapsed_ms(8, 9)
    ok_plain = all(np.array_equal(o.download(), w) for o, w in zip(outs, wants))
    # batched + learned: one persistent launch, sub-grid barriers, CUDA graph replay
    b = gsrb.Batch(ctx, dgs, gsrb.cfg(variant=gsrb.BAR_FANOUT, ctas_per_sm=2, threads=512, wake_lines=4))
    cg = gsrb.CudaGraph(ctx)
    with cg:
        gsrb.check(b.bfs([0] * 64, outs, gsrb.BFS_LEARNED), "batch bfs")
    for o in outs:
        o.zero()
    ts = []
    for rep in range(3):
        ctx.record(10)
        cg.launch()
        ctx.record(11)
        ts.append(ctx.elapsed_ms(10, 11))
    rc, st = b.stats()
    gsrb.check(rc, "batch stats")
    ok_batch = all(np.array_equal(o.download(), w) for o, w in zip(outs, wants))
    t_batch = statistics.median(ts)
    # the same batched launch with the fixed direction heuristic instead of the network
    cgh = gsrb.CudaGraph(ctx)
    with cgh:
        gsrb.check(b.bfs([0] * 64, outs, gsrb.BFS_HEURISTIC), "batch bfs heuristic")
    for o in outs:
        o.zero()
    tsh = []
    for rep in range(3):
        ctx.record(10)
        cgh.launch()
        ctx.record(11)
        tsh.append(ctx.elapsed_ms(10, 11))
    ok_heur = all(np.array_equal(o.download(), w) for o, w in zip(outs, wants))
    t_heur = statistics.median(tsh)
    cgh.free()
    res["bfs"] = {"plain_ms": round(t_plain, 3), "plain_GTEPS": round(m_total / (t_plain * 1e-3) / 1e9, 3),
                  "plain_bit_exact": ok_plain, "batched_learned_ms": round(t_batch, 3),
                  "batched_learned_GTEPS": round(m_total / (t_batch * 1e-3) / 1e9, 3),
                  "batched_learned_bit_exact": ok_batch, "speedup": round(t_plain / t_batch, 3),
                  "batched_heuristic_ms": round(t_heur, 3),
                  "batched_heuristic_GTEPS": round(m_total / (t_heur * 1e-3) / 1e9, 3),
                  "batched_heuristic_bit_exact": ok_heur,
                  "learned_vs_heuristic": round(t_heur / t_batch, 3),
                  "policy_decisions": int(sum(s.decisions for s in st)),
                  "fallbacks": int(sum(1 for s in st if s.aux))}
    cg.free()
    # SSSP: plain = one launch per graph with the reference's DELTA (10000);
    # batched = one launch with a tuned bucket width
    for rep in range(2):
        ctx.record(8)
        for dg, o in zip(dgs, outs):
            rc, _ = dg.sssp(0, o, 10000, plain_cfg)
            gsrb.check(rc, "plain sssp")
        ctx.record(9)
        t_plain = ctx.elapsed_ms(8, 9)
    ok_plain = all(np.array_equal(o.download(), w) for o, w in zip(outs, wants_d))
    def batched_sssp(delta):
        for o in outs:
            o.zero()
        ts = []
        for rep in range(3):
            ctx.record(10)
            gsrb.check(b.sssp([0] * 64, outs, delta), "batch sssp")
            ctx.record(11)
            ts.append(ctx.elapsed_ms(10, 11))
        rc, st = b.stats()
        gsrb.check(rc, "batch sssp stats")
        ok = all(np.array_equal(o.download(), w) for o, w in zip(outs, wants_d))
        return statistics.median(ts), ok, st

    t_fixed, ok_fixed, _ = batched_sssp(10000)
    t_256, ok_256, _ = batched_sssp(256)
    res["sssp"] = {"plain_ms": round(t_plain, 3), "plain_GTEPS": round(m_total / (t_plain * 1e-3) / 1e9, 3),
                   "plain_bit_exact": ok_plain,
                   "batched_fixed_delta_ms": round(t_fixed, 3),
                   "batched_fixed_delta_GTEPS": round(m_total / (t_fixed * 1e-3) / 1e9, 3),
                   "batched_delta256_ms": round(t_256, 3), "batched_bit_exact": ok_fixed and ok_256}
    t_best, ok_best = t_fixed, ok_fixed
    if sparams is not None:
        for dg in dgs:
            dg.set_sssp_policy(sparams)
        t_learn, ok_learn, st = batched_sssp(gsrb.SSSP_DELTA_LEARNED)
        res["sssp"].update({"batched_learned_ms": round(t_learn, 3),
                            "batched_learned_GTEPS": round(m_total / (t_learn * 1e-3) / 1e9, 3),
                            "batched_learned_bit_exact": ok_learn,
                            "learned_vs_fixed_delta": round(t_fixed / t_learn, 3),
                            "learned_deltas": sorted({int(x.delta) for x in st})})
        t_best, ok_best = t_learn, ok_learn
    res["sssp"].update({"batched_ms": round(t_best, 3), "batched_GTEPS": round(m_total / (t_best * 1e-3) / 1e9, 3),
                        "batched_bit_exact": res["sssp"]["batched_bit_exact"] and ok_best,
                        "speedup": round(t_plain / t_best, 3)})
    b.free()
    for dg in dgs:
        dg.free()
    return res


# ------------------------------------------------- the reference's GPU programs
REF_BIN = ROOT / "baseline" / "_ref"
_TIME_RE = [re.compile(r"average:\s*([0-9.eE+-]+)\s*ms"), re.compile(r"time \(ms\) is\s*([0-9.eE+-]+)"),
            re.compile(r"(?i)kernel time \(ms\)(?: is)?\s*([0-9.eE+-]+)"),
            re.compile(r"time cuda only\(ms\)\s*([0-9.eE+-]+)")]


def _ref_run(prog, args, stdin=None, timeout=180):
    """Runs one of the reference's own programs (recompiled for sm_100a) and
    returns (time in ms it printed, stdout).  Only co-resident shapes are
    passed: the GSRB forms spin without a bound."""
    # the program sees only this process's GPU (the LOCAL_RANK-th visible one)
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    local = int(os.environ.get("LOCAL_RANK", "0"))
    devs = [d for d in vis.split(",") if d] if vis else [str(local)]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES=devs[min(local, len(devs) - 1)] if vis else devs[0])
    p = subprocess.run([str(REF_BIN / prog)] + [str(a) for a in args], input=stdin, capture_output=True,
                       text=True, timeout=timeout, env=env)
    if p.returncode != 0:
        raise RuntimeError(f"{prog} rc {p.returncode}: {(p.stdout + p.stderr)[-300:]}")
    for rx in _TIME_RE:
        m = rx.search(p.stdout)
        if m:
            return float(m.group(1)), p.stdout
    raise RuntimeError(f"{prog}: no time in output")


# The reference's GSRB / GCPUSRB forms with more than one CTA per barrier group
# (more CTAs than SMs) measured slow on B200 in one run of this file: reduce at
# N = 303,104 (1184 CTAs of 256 threads) 8.5 s, scan at N = 151,552 (2368 CTAs
# of 32 threads) 15.8 s, Lonestar bfs_gsrb 38 s and sssp_gsrb 116 s on RMAT-22
# (block factor 2); on the 2048 x 2048 grid (4095 levels) bfs_gsrb and
# sssp_gsrb did not finish within 600 s and were killed.  The default run
# ("quick") times the reference's programs only at shapes that finish in
# seconds; "full" adds the slow RMAT-22, reduce and scan shapes.  The grid's
# GSRB / GCPUSRB forms are never run again.
REF_SLOW_SHAPES = {"reduce_gsrb_303104_ms": 8542.3, "scan_gsrb_151552_ms": 15834.8,
                   "rmat22_bfs_gsrb_ms": 38140.4, "rmat22_sssp_gsrb_ms": 115862.0,
                   "grid2048_bfs_gsrb": "not finished within 600 s (killed)",
                   "grid2048_sssp_gsrb": "not finished within 600 s (killed)"}


def reference_gpu_numbers(gsrb, ctx, mode="quick"):
    """The reference's own GPU programs (baseline/_ref, built from the
    reference sources for sm_100a by baseline/build.sh) timed on this GPU in
    the same run, beside this library on the same shapes.  Every shape is
    co-resident: Heterosync runs 148*k CTAs of 32 threads (k <= 8, the
    reference's own MAX_BLOCKS check allows 32 per SM), the reduce and scan run
    at N where one element per thread needs <= 8 CTAs per SM.  mode "quick"
    skips the GSRB forms at the shapes in REF_SLOW_SHAPES."""
    if not (REF_BIN / "allSyncPrims-1kernel").exists():
        return {"unavailable": "baseline/_ref not built (needs the reference sources)"}
    out = {"programs": "baseline/_ref, the reference's sources compiled for sm_100a", "mode": mode,
           "slow_shapes_recorded": REF_SLOW_SHAPES}
    iters = 10000 if mode == "full" else 1000
    # Heterosync barriers: one barrier per iteration, NUM_LDST = 1, 10 launches
    # averaged; quick mode at full residency only (each run of the program also
    # spends seconds in its cudaLocksInit, one cudaMemset per mutex word)
    het = []
    for k in ((1, 8) if mode == "full" else (8,)):
        ntb = 148 * k
        row = {"ctas": ntb, "threads": 32, "iterations": iters}
        for name, prim in (("gsrb", "atomicTreeBarrUniqSRB"), ("gcpusrb", "atomicTreeBarrUniqNaiveSRB"),
                           ("ccg", "atomicTreeBarrUniqCCG"), ("atomic_tree", "atomicTreeBarrUniq")):
            try:
                ms, _ = _ref_run("allSyncPrims-1kernel", [prim, 1, ntb, iters])
                row[name + "_ns"] = round(ms * 1e6 / iters, 1)
            except Exception as e:  # noqa: BLE001
                row[name + "_ns"] = f"failed: {str(e)[:120]}"
        # this library on the same shape (32-thread CTAs, F = 0), its own protocols
        for name, v in (("native_fanout", gsrb.BAR_FANOUT), ("native_flip", gsrb.BAR_FLIP)):
            c = gsrb.cfg(variant=v, ctas_per_sm=k, threads=32, wake_lines=2)
            none = gsrb.cfg(variant=gsrb.BAR_NONE, ctas_per_sm=k, threads=32)
            t0 = statistics.median(time_barrier(gsrb, ctx, none, 2000, 0, 3, 1))
            t1 = statistics.median(time_barrier(gsrb, ctx, c, 2000, 0, 3, 1))
            row[name + "_ns"] = round((t1 - t0) * 1e6 / 2000, 1)
        het.append(row)
    out["heterosync_barrier"] = het

    def native_time(fn):
        ts = []
        for i in range(8):
            ctx.record(4)
            fn()
            ctx.record(5)
            if i >= 3:
                ts.append(ctx.elapsed_ms(4, 5))
        return round(statistics.median(ts), 5)

    # reduce: one element per thread, 256 threads per CTA
    red = []
    for n in (37_888, 303_104):
        row = {"n": n}
        for v in ("gsrb", "ccg"):
            if v == "gsrb" and n > 37_888 and mode != "full":
                row[v + "_ms"] = f"not run (measured {REF_SLOW_SHAPES['reduce_gsrb_303104_ms']} ms once)"
                continue
            try:
                ms, so = _ref_run(f"reduce_{v}", [n, 256])
                row[v + "_ms"] = ms
                row[v + "_correct"] = f"Sum: {n}\n" in so
            except Exception as e:  # noqa: BLE001
                row[v + "_ms"] = f"failed: {str(e)[:120]}"
        a = np.ones(n, np.int32)
        d = ctx.to_device(a)
        o = ctx.array(1, np.int64).zero()
        row["native_ms"] = native_time(lambda: gsrb.check(ctx.reduce_i32(d, n, o)))
        row["native_correct"] = int(o.download()[0]) == n
        d.free()
        o.free()
        red.append(row)
    out["reduce"] = red
    # scan: 64-element tiles of 32-thread CTAs
    scn = []
    for n in (9_472, 151_552):
        row = {"n": n}
        for v in ("gsrb", "ccg"):
            if v == "gsrb" and n > 9_472 and mode != "full":
                row[v + "_ms"] = f"not run (measured {REF_SLOW_SHAPES['scan_gsrb_151552_ms']} ms once)"
                continue
            try:
                ms, so = _ref_run(f"scan_{v}", [n])
                row[v + "_ms"] = ms
                row[v + "_match"] = "Match: 1" in so
            except Exception as e:  # noqa: BLE001
                row[v + "_ms"] = f"failed: {str(e)[:120]}"
        a = np.ones(n, np.uint32)
        d, o = ctx.to_device(a), ctx.array(n, np.uint32)
        row["native_ms"] = native_time(lambda: gsrb.check(ctx.scan(d, o, n)))
        row["native_match"] = bool(np.array_equal(o.download(), np.arange(n, dtype=np.uint32)))
        d.free()
        o.free()
        scn.append(row)
    out["scan"] = scn
    return out


def lonestar_reference(g, name, mode="quick", timeout=300):
    """The reference's Lonestar BFS and SSSP on graph g written as .gr v1: the
    "Kernel time (ms)" each prints, block factor 2 (296 CTAs of 32 threads,
    within the wrapper's own residency cap).  The cooperative-groups builds
    always; the GSRB builds only in mode "full" and never on the grid (see
    REF_SLOW_SHAPES)."""
    if not (REF_BIN / "lonestar" / "bfs_gsrb").exists():
        return {"unavailable": "baseline/_ref not built (needs the reference sources)"}
    row = {"block_factor": 2}
    with tempfile.TemporaryDirectory() as td:
        path = pathlib.Path(td) / "g.gr"
        g.write_gr(path, with_weights=True)
        for app, extra in (("bfs", ["-s", 0]), ("sssp", ["-s", 0, "-d", 10000])):
            for v in ("gsrb", "ccg"):
                if v == "gsrb" and (mode != "full" or name != "rmat22"):
                    row[f"{app}_{v}_ms"] = f"not run: {REF_SLOW_SHAPES.get(f'{name}_{app}_gsrb_ms', REF_SLOW_SHAPES.get(f'{name}_{app}_gsrb'))}"
                    continue
                try:
                    ms, _ = _ref_run(f"lonestar/{app}_{v}", extra + ["-q", path], stdin="2\n", timeout=timeout)
                    row[f"{app}_{v}_ms"] = ms
                except Exception as e:  # noqa: BLE001
                    row[f"{app}_{v}_ms"] = f"failed: {str(e)[:120]}"
    return row


def cpu_barrier_baseline(orc, nctas, seconds=8.0):
    """The reference's two-level sense-reversing barrier restated on the host
    cores, with the same participants as the GPU workload: `nctas` CTAs in
    min(nctas, 148) groups (CTA % 148, as the reference groups by blockIdx %
    NUM_SM), carried by one thread per core, each arriving for its CTAs in turn."""
    threads = os.cpu_count() or 1
    groups = min(nctas, 148)
    ns, stale = orc.cpu_srb_barrier_vcta(threads, nctas, groups, 200)
    episodes = int(max(200, min(5_000_000, seconds * 1e9 / max(ns, 1.0) / 2)))
    ns, stale = orc.cpu_srb_barrier_vcta(threads, nctas, groups, episodes)
    return {"value": round(ns, 2), "unit": "ns per barrier", "cores": threads, "kind": "port",
            "sample": f"{nctas} CTAs (the GPU workload's) carried by {threads} host threads, one per core, "
                      f"{groups} groups, {2 * episodes} barrier episodes, F=0, stale reads {stale}"}


# --------------------------------------------------------------- the summary
def _get(d, *keys):
    for k in keys:
        if not isinstance(d, dict) or k not in d:
            return None
        d = d[k]
    return d


def tail_summary(cf):
    """The headline figures of every configuration in a few hundred bytes; the
    JSON line ends with it, so a reader that keeps only the line's tail still
    sees them (the full entries are in "configs" and in the detail file)."""
    def g(d, *ks):
        for k in ks:
            d = d.get(k) if isinstance(d, dict) else None
        return d
    c1, c3 = cf.get("C1_reduce_2e24") or {}, cf.get("C3_scan_2e28") or {}
    rm, gd = cf.get("C4_rmat22") or {}, cf.get("C4_grid2048") or {}
    b5, s5 = cf.get("C5_batch64") or {}, cf.get("C5_segments64") or {}
    sem = cf.get("C2_semaphore") or {}
    return {
        "C1_reduce": {"us": c1.get("us"), "hbm_frac": c1.get("hbm_frac"), "unchained_hbm_frac": c1.get("unchained_hbm_frac"),
                      "cold_single_us": c1.get("single_launch_cold_us"), "exact": c1.get("bit_exact"),
                      "cpu_mt_GB_s": c1.get("cpu_mt_GB_s")},
        "C2_barrier_k8_x_ccg": {k: g(v, "x_ccg") for k, v in (cf.get("C2_barrier_k8") or {}).items()},
        "C2_ref_programs_k8_ns": g(cf, "C2_barrier_reference_programs", "k8"),
        "C2_sem_acq_per_s": {k: g(v, "acq_per_s") for k, v in sem.items()},
        "C3_scan": {"u32_hbm_frac": c3.get("u32_hbm_frac"), "f32_hbm_frac": c3.get("f32_hbm_frac"),
                    "exact": c3.get("u32_bit_exact"), "cpu_mt_GB_s": c3.get("cpu_mt_GB_s")},
        "C4_rmat22": {"bfs_GTEPS": rm.get("bfs_learned_GTEPS"), "bfs_x_plain": rm.get("bfs_learned_vs_plain"),
                      "sssp_GTEPS": rm.get("sssp_GTEPS"), "pr_frac_gather_floor": rm.get("pr_frac_of_gather_floor"),
                      "exact": bool(rm.get("bfs_bit_exact") and rm.get("sssp_bit_exact"))},
        "C4_grid2048_ms": {"bfs": gd.get("bfs_heuristic_ms"), "sssp": gd.get("sssp_ms")},
        "C5_batch64": {"bfs_x_plain": b5.get("bfs_learned_vs_plain"), "bfs_x_heuristic": b5.get("bfs_learned_vs_heuristic"),
                       "sssp_x_plain": b5.get("sssp_speedup"), "exact": b5.get("bit_exact")},
        "C5_segments64_hbm_frac": {"reduce": s5.get("reduce_hbm_frac"), "scan": s5.get("scan_hbm_frac")},
    }


def summarize(detail, peak):
    """One compact entry per benchmark configuration for the JSON line (the
    full tables go to the detail file): time, throughput, roofline fraction of
    measured HBM where the kernel is HBM-bound, correctness, and the CPU
    baseline of the same workload."""
    out = {}
    bt = detail.get("barrier_table") or []
    out["C2_barrier_k8"] = {f"F{r['F']}": {"native_ns": r.get("native"), "ccg_ns": r.get("ccg"),
                                           "x_ccg": r.get("speedup_vs_ccg"), "variant": r.get("tuned")}
                            for r in bt if r.get("k") == 8}
    rg = detail.get("reference_gpu") or {}
    if "heterosync_barrier" in rg:
        out["C2_barrier_reference_programs"] = {f"k{r['ctas'] // 148}": {k: v for k, v in r.items() if k.endswith("_ns")}
                                                for r in rg["heterosync_barrier"]}
    sem = (detail.get("semaphore") or {}).get("rows") or []
    out["C2_semaphore"] = {f"S{r['S']}": {"acq_per_s": _get(r, "native_priority", "acquires_per_s"),
                                          "x_serial_holds": _get(r, "native_priority", "x_serial_holds"),
                                          "ref_protocol_acq_per_s": _get(r, "ref_priority", "acquires_per_s"),
                                          "ref_spin_acq_per_s": _get(r, "ref_spin", "acquires_per_s"),
                                          "exact": _get(r, "native_priority", "exact")} for r in sem}
    r = detail.get("reduce_2e24") or {}
    out["C1_reduce_2e24"] = {"us": round(r["ms"] * 1e3, 2) if "ms" in r else None, "GB_s": r.get("GB_s"),
                             "hbm_frac": r.get("hbm_frac"), "bit_exact": r.get("bit_exact"),
                             "variant": _get(r, "cfg", "variant"), "shape": "148x2x256",
                             "ccg_us": round(r["ccg_ms"] * 1e3, 2) if r.get("ccg_ms") else None,
                             "chained": bool(_get(r, "cfg", "overlap")),
                             "unchained_us": round(r["unchained"]["ms"] * 1e3, 2) if r.get("unchained") else None,
                             "unchained_hbm_frac": _get(r, "unchained", "hbm_frac"),
                             "tuned_any_shape_hbm_frac": _get(r, "tuned_any_shape", "hbm_frac"),
                             "single_launch_cold_us": r.get("single_launch_cold_us"),
                             "dram_traffic_per_launch": profile_traffic(
                                 "reduce_i32_kernel_2e24_chained" if _get(r, "cfg", "overlap")
                                 else "reduce_i32_kernel_2e24"),
                             "cpu_serial_GB_s": _get(r, "cpu", "serial_GB_s"), "cpu_mt_GB_s": _get(r, "cpu", "mt_GB_s")}
    if "reduce" in rg:
        out["C1_reduce_reference_programs"] = rg["reduce"]
    sc = detail.get("scan_2e28") or {}
    out["C3_scan_2e28"] = {"u32_ms": _get(sc, "u32", "ms"), "u32_hbm_frac": _get(sc, "u32", "hbm_frac"),
                           "u32_bit_exact": _get(sc, "u32", "bit_exact"), "f32_ms": _get(sc, "f32", "ms"),
                           "f32_hbm_frac": _get(sc, "f32", "hbm_frac"), "f32_max_rel_err": _get(sc, "f32", "max_rel_err"),
                           "cpu_ref_serial_GB_s": _get(sc, "cpu", "serial_GB_s"), "cpu_mt_GB_s": _get(sc, "cpu", "mt_GB_s")}
    if "scan" in rg:
        out["C3_scan_reference_programs"] = rg["scan"]
    gr = detail.get("graphs") or {}
    for key, name in (("rmat22", "C4_rmat22"), ("grid2048", "C4_grid2048")):
        g = gr.get(key) or {}
        b = g.get("bfs") or {}
        n, m = g.get("n"), g.get("m")
        e = {"n": n, "m": m}
        for arm in ("plain_push", "heuristic", "learned"):
            e[f"bfs_{arm}_ms"] = _get(b, arm, "ms")
            e[f"bfs_{arm}_GTEPS"] = _get(b, arm, "GTEPS")
        if _get(b, "heuristic", "ms") and _get(b, "learned", "ms"):
            e["bfs_learned_vs_heuristic"] = round(b["heuristic"]["ms"] / b["learned"]["ms"], 3)
            e["bfs_learned_vs_plain"] = round(b["plain_push"]["ms"] / b["learned"]["ms"], 3)
        if n and m and _get(b, "heuristic", "ms"):
            # one traversal's algorithmic bytes: row offsets, edges, level writes
            byts = 4 * (n + 1) + 4 * m + 4 * n
            e["bfs_heuristic_hbm_frac"] = round(byts / (b["heuristic"]["ms"] * 1e-3) / 1e9 / peak, 4)
        e["bfs_bit_exact"] = all(_get(b, a, "bit_exact") for a in ("plain_push", "heuristic", "learned"))
        ss = g.get("sssp") or {}
        first = next((v for k, v in ss.items() if k != "cpu"), {})
        e["sssp_ms"], e["sssp_GTEPS"], e["sssp_bit_exact"] = first.get("ms"), first.get("GTEPS"), first.get("bit_exact")
        pr = g.get("pagerank") or {}
        if pr:
            e["pr50_ms"], e["pr_hbm_frac"], e["pr_l1"] = pr.get("ms"), pr.get("hbm_frac"), pr.get("l1_vs_fp64")
            e["pr_frac_of_gather_floor"] = _get(g, "pagerank_gather_floor", "frac_of_gather_floor")
            e["pr_gather_floor_hbm_frac"] = _get(g, "pagerank_gather_floor", "floor_hbm_frac")
        e["cpu_bfs_serial_GTEPS"] = _get(b, "cpu", "serial_GTEPS")
        e["cpu_bfs_mt_GTEPS"] = _get(b, "cpu", "mt_GTEPS")
        e["cpu_sssp_serial_GTEPS"] = _get(ss, "cpu", "serial_GTEPS")
        if pr:
            e["cpu_pr_serial_ms_per_iter"] = _get(pr, "cpu", "serial_ms_per_iter")
            e["cpu_pr_mt_ms_per_iter"] = _get(pr, "cpu", "mt_ms_per_iter")
        ref = g.get("reference_gpu")
        if ref:
            e["reference_programs_ms"] = ref
        out[name] = e
    bb = detail.get("batch") or {}
    out["C5_batch64"] = {"bfs_plain_GTEPS": _get(bb, "bfs", "plain_GTEPS"),
                         "bfs_batched_heuristic_GTEPS": _get(bb, "bfs", "batched_heuristic_GTEPS"),
                         "bfs_batched_learned_GTEPS": _get(bb, "bfs", "batched_learned_GTEPS"),
                         "bfs_learned_vs_plain": _get(bb, "bfs", "speedup"),
                         "bfs_learned_vs_heuristic": _get(bb, "bfs", "learned_vs_heuristic"),
                         "sssp_plain_GTEPS": _get(bb, "sssp", "plain_GTEPS"),
                         "sssp_batched_GTEPS": _get(bb, "sssp", "batched_GTEPS"),
                         "sssp_speedup": _get(bb, "sssp", "speedup"),
                         "bit_exact": all(_get(bb, *k) for k in (("bfs", "plain_bit_exact"),
                                                                 ("bfs", "batched_learned_bit_exact"),
                                                                 ("bfs", "batched_heuristic_bit_exact"),
                                                                 ("sssp", "batched_bit_exact"))),
                         "cpu_bfs_mt_GTEPS": _get(bb, "cpu", "bfs_mt_GTEPS"),
                         "cpu_sssp_mt_GTEPS": _get(bb, "cpu", "sssp_mt_GTEPS")}
    sg = detail.get("segments") or {}
    out["C5_segments64"] = {"reduce_hbm_frac": _get(sg, "reduce", "batched_hbm_frac"),
                            "reduce_x_per_segment": _get(sg, "reduce", "speedup_vs_per_segment_graph"),
                            "scan_hbm_frac": _get(sg, "scan", "batched_hbm_frac"),
                            "scan_x_per_segment": _get(sg, "scan", "speedup_vs_per_segment_graph"),
                            "bit_exact": bool(_get(sg, "reduce", "bit_exact") and _get(sg, "scan", "bit_exact"))}
    pol = detail.get("policy") or {}
    out["policy"] = {k: pol.get(k) for k in ("levels", "train_s", "loss_first", "loss_last") if k in pol}
    return out


def profile_traffic(name):
    """DRAM bytes per launch recorded in a kept ncu summary (profiles/<name>.md,
    the line 'traffic_bytes_per_launch: N'), or None."""
    try:
        m = re.search(r"traffic_bytes_per_launch:\s*([0-9]+)", (ROOT / "profiles" / f"{name}.md").read_text())
        return int(m.group(1)) if m else None
    except OSError:
        return None


# ----------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="barrier", choices=["barrier", "reduce", "scan", "segments", "bfs", "sssp", "pr",
                                                              "prr"])
    ap.add_argument("--graph", default="rmat", choices=["rmat", "grid"], help="graph of the bfs/sssp/pr workloads")
    ap.add_argument("--scale", type=int, default=22, help="log2 vertices of the bfs/sssp/pr workload graph")
    ap.add_argument("--iters", type=int, default=50, help="PageRank iterations (pr workload)")
    ap.add_argument("--delta", type=int, default=10000, help="SSSP bucket width (sssp workload)")
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--fma", type=int, default=0)
    ap.add_argument("--cfg", type=json.loads, default=None,
                    help="fixed configuration as JSON (skips the autotuner), e.g. '{\"variant\": 9}'")
    ap.add_argument("--episodes", type=int, default=10_000)
    ap.add_argument("--scan-n", type=int, default=1 << 28)
    ap.add_argument("--reduce-n", type=int, default=1 << 24)
    ap.add_argument("--no-extras", action="store_true")
    ap.add_argument("--skip-pr-check", action="store_true", help="skip the FP64 CPU PageRank (about 25 s)")
    ap.add_argument("--reference-programs", default="quick", choices=["none", "quick", "full"],
                    help="time the reference's own GPU programs (baseline/_ref): quick = the shapes that finish "
                         "in seconds, full = also the slow GSRB shapes (minutes)")
    ap.add_argument("--detail", default=str(ROOT / "gpurun_out" / "bench_detail.json"),
                    help="where the full tables go (the JSON line keeps one summary per configuration)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    dist = Dist()
    base_cfg = {"workload": f"grid barrier microbenchmark: 148*{args.k} CTAs x 256 threads, "
                            f"{args.episodes} episodes per launch, F={args.fma} FMAs/thread/episode",
                "ctas": 148 * args.k, "threads_per_cta": 256, "episodes_per_step": args.episodes,
                "fma_per_episode": args.fma, "parallelism": f"replicas x{args.gpus}",
                "l2": "read-flushed (2x L2) before every timed launch"}

    if args.impl == "reference":
        if dist.rank == 0:
            orc = load_oracle()
            t0 = time.time()
            for _ in range(args.warmup):  # untimed warm-up samples
                cpu_barrier_baseline(orc, 148 * args.k, seconds=0.2)
            samples = [cpu_barrier_baseline(orc, 148 * args.k, seconds=2.0) for _ in range(max(1, args.steps))]
            v = statistics.median(s["value"] for s in samples)
            line = {"impl": "reference", "metric": "ns per grid barrier", "value": v, "unit": "ns",
                    "n_gpus": args.gpus, "steps": len(samples), "warmup": args.warmup,
                    "ms_per_step": round((time.time() - t0) * 1e3 / len(samples), 2),
                    "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                    "data": "synthetic", "config": base_cfg,
                    "cpu_baseline": dict(samples[0], value=v),
                    "e2e": {"value": v, "unit": "ns", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
            print(json.dumps(line), flush=True)
        dist.close()
        return

    gsrb = load_binding()
    tune = _load("gsrb_autotune", PKG / "autotune.py")
    ctx = gsrb.Context(dist.local if dist.world > 1 else 0)
    cache = {}

    if args.workload != "barrier":
        # single data-kernel workloads (profiling entry points)
        orc = load_oracle()
        if args.workload == "reduce":
            r = reduce_numbers(gsrb, ctx, orc, tune, cache, reps=args.steps, fixed=args.cfg, n=args.reduce_n)
        elif args.workload == "scan":
            r = scan_numbers(gsrb, ctx, orc, tune, cache, n=args.scan_n, reps=args.steps, fixed=args.cfg)
        elif args.workload == "segments":
            r = segment_numbers(gsrb, ctx, orc, tune, cache, reps=args.steps, fixed=args.cfg)
        else:
            g = (gsrb.grid2d(1 << (args.scale // 2), 1 << (args.scale - args.scale // 2), seed=SEED)
                 if args.graph == "grid" else gsrb.rmat(args.scale, 16, seed=SEED))
            dg = ctx.graph(g)
            c = tune.cfg_from(args.cfg) if args.cfg else None
            if args.workload == "bfs":
                r = bfs_runs(gsrb, ctx, orc, dg, g, gsrb.mlp_init(1), c, reps=args.steps)
            elif args.workload == "sssp":
                r = sssp_runs(gsrb, ctx, orc, dg, g, [("delta", args.delta)], c)
            elif args.workload == "prr":
                # the reference's push-residual PageRank (epsilon 1e-6, to an empty worklist)
                out = ctx.array(g.nnodes, np.float32)
                ts = []
                for _ in range(args.steps):
                    rc, st = dg.pagerank_residual(out, 0.85, 1e-6, 2**31 - 1, c)
                    gsrb.check(rc, "pagerank_residual")
                    ts.append(st.kernel_ms)
                r = {"n": g.nnodes, "m": g.nedges, "ms": ts, "rounds": int(st.levels), "pushes": int(st.edges)}
            else:
                out = ctx.array(g.nnodes, np.float32)
                ts = []
                for _ in range(args.steps):
                    rc, st = dg.pagerank(out, 0.85, args.iters, c)
                    gsrb.check(rc, "pagerank")
                    ts.append(st.kernel_ms)
                l1 = orc.normalized_l1(out.download(), orc.pagerank(g, 0.85, args.iters))
                r = {"n": g.nnodes, "m": g.nedges, "iters": args.iters, "ms": ts, "l1_vs_fp64": l1}
            dg.free()
        if dist.rank == 0:
            print(json.dumps({"workload": args.workload, "result": r}), flush=True)
        ctx.close()
        dist.close()
        return

    if args.cfg:
        best, tune_table = dict(args.cfg, ctas_per_sm=args.k, threads=256), []
    else:
        best, _, tune_table = tune.tune_barrier(ctx, args.k, episodes=2000, reps=2)
    cache[f"barrier_k{args.k}"] = best
    c = tune.cfg_from(best)
    none = gsrb.cfg(variant=gsrb.BAR_NONE, ctas_per_sm=args.k, threads=256)
    t_phase = statistics.median(time_barrier(gsrb, ctx, none, args.episodes, args.fma, 5, 3))

    clocks = Clocks(ctx.device)
    dist.barrier()
    ctx.sync()
    clocks.start()
    l0 = gsrb.launch_count()
    times = time_barrier(gsrb, ctx, c, args.episodes, args.fma, args.steps, args.warmup)
    l1 = gsrb.launch_count()
    ctx.sync()
    clk = clocks.stop()
    dist.barrier()

    t_step = statistics.median(times)
    ns = dist.max((t_step - t_phase) * 1e6 / args.episodes)
    ms_per_step = dist.max(statistics.mean(times))
    e2e_times, bi, bo = barrier_e2e(gsrb, ctx, c, args.episodes, args.fma, 5, 3)
    e2e_ns = dist.max(statistics.median(e2e_times) * 1e6 / args.episodes)
    t_ccg = statistics.median(time_barrier(gsrb, ctx, gsrb.cfg(variant=gsrb.BAR_CCG, ctas_per_sm=args.k,
                                                              threads=256), args.episodes, args.fma, 5, 2))
    ns_ccg = (t_ccg - t_phase) * 1e6 / args.episodes

    rate, rtt = l2_atomic_peak(ctx)
    grid = args.k * ctx.num_sms
    arrivals = arrivals_per_episode(gsrb, c, grid)
    achieved = arrivals / (ns * 1e-9)
    # DRAM bytes of one launch from the kept ncu capture of this kernel (1184 x
    # 256, F = 0): the per-thread FMA seeds, read once, independent of episodes
    traffic = profile_traffic("barrier_bench_kernel_fanout_k8") if args.k == 8 and args.fma == 0 else None
    roofline = {"bound": "l2_atomic", "achieved": round(achieved / 1e9, 4), "peak": round(rate / 1e9, 4),
                "unit": "G same-address atomics/s", "frac": round(achieved / rate, 4), "traffic": traffic,
                "traffic_note": "dram__bytes_read.sum + dram__bytes_write.sum per launch (ncu); the barrier is "
                                "L2-latency bound, DRAM idle",
                "peak_source": "measured live: same-address red.add throughput probe (MEASURED_PEAKS.json has no "
                               "L2-atomic entry)",
                "arrivals_per_episode": arrivals, "l2_atomic_rtt_ns": round(rtt, 1),
                "latency_floor_ns": round(arrivals / rate * 1e9 + 2 * rtt, 1),
                "latency_floor_frac": round((arrivals / rate * 1e9 + 2 * rtt) / ns, 4)}

    line = {"metric": "ns per grid barrier", "value": round(ns, 2), "unit": "ns", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": dict(base_cfg, barrier=gsrb.VARIANT_NAMES[c.variant], tuned=best),
            "phase_only_ms": round(t_phase, 5), "ccg_grid_sync_ns": round(ns_ccg, 2),
            "speedup_vs_ccg": round(ns_ccg / ns, 3), "roofline": roofline, "clocks": clk,
            "gpu_launches": int(l1 - l0),
            "e2e": {"value": round(e2e_ns, 2), "unit": "ns", "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                    "note": "per-episode time of the whole step incl. pinned H2D/D2H copies and the FMA phase"},
            }
    detail = {"headline": dict(line), "autotune_top5": [{"ns": t, "cfg": cand} for t, cand in tune_table[:5]]}

    # the other configurations are measured at one GPU only: with N > 1 every
    # GPU would repeat them (replicas) while all N are held
    if not args.no_extras and dist.world == 1:
        orc = load_oracle()
        pol = _load("gsrb_policy", PKG / "policy.py")
        extras_t0 = time.time()
        walls = {}

        def timed(key, fn):
            t = time.time()
            r = fn()
            walls[key] = round(time.time() - t, 1)
            return r

        detail["barrier_table"] = timed("barrier_table", lambda: barrier_table(gsrb, ctx, tune, cache))
        detail["semaphore"] = timed("semaphore", lambda: semaphore_numbers(gsrb, ctx))
        detail["reduce_2e24"] = timed("reduce", lambda: reduce_numbers(gsrb, ctx, orc, tune, cache,
                                                                       cpu=dist.rank == 0))
        detail["scan_2e28"] = timed("scan", lambda: scan_numbers(gsrb, ctx, orc, tune, cache, n=args.scan_n,
                                                                 cpu=dist.rank == 0))
        params, pinfo = timed("policy", lambda: train_policy(gsrb, ctx, pol))
        detail["policy"] = pinfo
        sparams, spinfo = timed("sssp_policy", lambda: train_sssp_policy(gsrb, ctx, pol))
        detail["sssp_policy"] = spinfo
        detail["graphs"] = timed("graphs", lambda: graph_numbers(gsrb, ctx, orc, pol, params, sparams, tune, cache,
                                                                 not args.skip_pr_check,
                                                                 ref_gpu=args.reference_programs))
        detail["batch"] = timed("batch", lambda: batch_numbers(gsrb, ctx, orc, params, sparams))
        detail["segments"] = timed("segments", lambda: segment_numbers(gsrb, ctx, orc, tune, cache))
        if args.reference_programs != "none":
            detail["reference_gpu"] = timed("reference_programs",
                                            lambda: reference_gpu_numbers(gsrb, ctx, args.reference_programs))
        detail["wall_s"] = walls
        line["extras_wall_s"] = round(time.time() - extras_t0, 1)
        line["extras_walls"] = walls
        line["configs"] = summarize(detail, hbm_peak()[0])
        if dist.rank == 0:
            line["cpu_baseline"] = cpu_barrier_baseline(orc, 148 * args.k)
    detail["autotuned"] = cache

    if dist.rank == 0:
        try:
            dpath = pathlib.Path(args.detail)
            dpath.parent.mkdir(parents=True, exist_ok=True)
            dpath.write_text(json.dumps(detail, indent=1, default=str))
            line["detail_file"] = str(args.detail)
        except OSError as e:
            line["detail_file"] = f"not written: {e}"
        if "configs" in line:
            line["summary"] = tail_summary(line["configs"])
        print(json.dumps(line), flush=True)
    ctx.close()
    dist.close()


if __name__ == "__main__":
    main()
