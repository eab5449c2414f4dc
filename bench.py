#!/usr/bin/env python
"""Benchmark driver: one JSON line on rank 0.

Headline workload (the configuration the metric is quoted on): the grid-barrier
microbenchmark -- one persistent launch of 148*k CTAs x 256 threads running
10,000 barrier episodes (k = 8: full residency, 2048 threads per SM), each
episode preceded by F dependent FP32 FMAs per thread (F = 0 for the headline).
value = ns per grid barrier = (t_launch - t_phase_only) / episodes, lower is
better.  The line also carries the data-phase kernels measured on the same
device: reduce (2^24 int32) and scan (2^28 u32 / f32) GB/s against the measured
HBM peak, and the comparison barriers (cooperative-groups grid.sync, the
reference GSRB/GCPUSRB/atomic-tree algorithms) on the same shape.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload barrier|reduce|scan] [--k 8] [--fma 0]

--impl reference times the reference's CPU implementation of the path on the
host cores (the reference has no CPU barrier, so this is the oracle port of
its sense-reversing barrier run by host threads), same metric and unit.
Multi-GPU: the barrier does not shard (replicas only): every rank runs the same
workload on its own GPU and the reported time is the max over ranks.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0


def load_binding():
    spec = importlib.util.spec_from_file_location("gsrb_b200", ROOT / "tpds22-artifact_b200" / "gsrb.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gsrb_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle_binding  # noqa: E402  (CPU baseline leg only)
    return oracle_binding


def hbm_peak():
    try:
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback 6.65 TB/s"


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
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
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


# ------------------------------------------------------------------ workloads
def best_native_cfg(gsrb, ctx, k, threads=256):
    """The native three-level barrier configuration used for the headline.

    Cluster 8 with a fan-in layer keeps the global counter at <= 37 arrivals;
    falls back to smaller clusters when the device cannot co-schedule it."""
    for cl, fan in ((8, 0), (4, 0), (2, 0), (1, 0)):
        c = gsrb.cfg(variant=gsrb.BAR_CLUSTER if cl > 1 else gsrb.BAR_SOFT2, ctas_per_sm=k, threads=threads,
                     cluster=cl, fanin_groups=fan)
        try:
            if ctx.max_coresident(c, 0) >= k * ctx.num_sms:
                return c
        except gsrb.GsrbError:
            continue
    return gsrb.cfg(variant=gsrb.BAR_FLAT, ctas_per_sm=k, threads=threads)


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
    """Same launch through the public C ABI with host buffers: H2D of the
    per-thread FMA state (pinned), the persistent launch, D2H of the results."""
    import ctypes as C
    lib = gsrb.lib()
    grid = c.ctas_per_sm * ctx.num_sms
    n = grid * c.threads
    h_in = C.c_void_p()
    h_out = C.c_void_p()
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


def l2_atomic_peak(gsrb, ctx):
    """Same-address red.add throughput (atomics/s) and atom round trip (ns)."""
    ctas, iters = 4 * ctx.num_sms, 2000
    ctx.probe_l2_atomics(ctas, 200, 0)
    ms = min(ctx.probe_l2_atomics(ctas, iters, 0) for _ in range(3))
    rate = ctas * iters / (ms * 1e-3)
    ctx.probe_l2_atomics(1, 1000, 1)
    ms1 = min(ctx.probe_l2_atomics(1, 20000, 1) for _ in range(3))
    rtt_ns = ms1 * 1e6 / 20000
    return rate, rtt_ns


def reduce_numbers(gsrb, ctx, orc, reps=10):
    n = 1 << 24
    a = gsrb.uniform_i32(0x5EED2022, n, 0, 127)
    d = ctx.to_device(a)
    out = ctx.array(1, np.int64).zero()
    c = gsrb.cfg(ctas_per_sm=2, threads=256, cluster=2)
    times = []
    for i in range(3 + reps):
        ctx.l2_flush()  # 64 MiB fits in L2: time it cold
        ctx.record(4)
        gsrb.check(ctx.reduce_i32(d, n, out, c))
        ctx.record(5)
        if i >= 3:
            times.append(ctx.elapsed_ms(4, 5))
    ctx.check_status("reduce")
    ok = int(out.download()[0]) == orc.sum_i32(a)
    t = statistics.median(times)
    gbs = 4 * n / (t * 1e-3) / 1e9
    d.free()
    return {"n": n, "ms": round(t, 5), "GB_s": round(gbs, 1), "bit_exact": ok, "cold_l2": True}


def cpu_barrier_baseline(orc, seconds=8.0):
    threads = os.cpu_count() or 1
    groups = 0 if threads <= 4 else max(2, threads // 4)
    ns, stale = orc.cpu_srb_barrier(threads, groups, 2000)
    episodes = int(max(2000, min(5_000_000, seconds * 1e9 / max(ns, 1.0) / 2)))
    ns, stale = orc.cpu_srb_barrier(threads, groups, episodes)
    return {"value": round(ns, 2), "unit": "ns per barrier", "cores": threads, "kind": "port",
            "sample": f"{threads} host threads (one per core standing in for the 1184 CTAs), "
                      f"{groups} groups, {2 * episodes} barrier episodes, stale reads {stale}"}


# ----------------------------------------------------------------------- main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="barrier", choices=["barrier"])
    ap.add_argument("--k", type=int, default=8)
    ap.add_argument("--fma", type=int, default=0)
    ap.add_argument("--episodes", type=int, default=10_000)
    ap.add_argument("--no-extras", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    dist = Dist()
    base_cfg = {"workload": f"grid barrier microbenchmark: 148*{args.k} CTAs x 256 threads, "
                            f"{args.episodes} episodes per launch, F={args.fma} FMAs/thread/episode",
                "ctas": 148 * args.k, "threads_per_cta": 256, "episodes_per_step": args.episodes,
                "fma_per_episode": args.fma, "parallelism": f"replicas x{args.gpus}",
                "l2": "flushed (write of 2x L2) before every timed launch"}

    if args.impl == "reference":
        if dist.rank == 0:
            orc = load_oracle()
            res = []
            for _ in range(args.warmup):
                pass
            t0 = time.time()
            samples = [cpu_barrier_baseline(orc, seconds=4.0) for _ in range(max(1, min(args.steps, 3)))]
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
    ctx = gsrb.Context(dist.local if dist.world > 1 else 0)
    c = best_native_cfg(gsrb, ctx, args.k)
    none = gsrb.cfg(variant=gsrb.BAR_NONE, ctas_per_sm=args.k, threads=256)

    # phase-only baseline (same launch, no barrier)
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
    ns_local = (t_step - t_phase) * 1e6 / args.episodes
    ns = dist.max(ns_local)
    ms_per_step = dist.max(statistics.mean(times))

    e2e_times, bi, bo = barrier_e2e(gsrb, ctx, c, args.episodes, args.fma, 5, 3)
    e2e_ns = dist.max(statistics.median(e2e_times) * 1e6 / args.episodes)

    rate, rtt = l2_atomic_peak(gsrb, ctx)
    grid = args.k * ctx.num_sms
    arrivals = grid // max(1, c.cluster) if c.variant in (0, 1, 2, 7) else grid
    achieved = arrivals / (ns * 1e-9)  # global-level atomics per second
    roofline = {"bound": "l2_atomic", "achieved": round(achieved / 1e9, 4), "peak": round(rate / 1e9, 4),
                "unit": "G same-address atomics/s", "frac": round(achieved / rate, 4), "traffic": None,
                "peak_source": "measured live: same-address red.add throughput probe",
                "arrivals_per_episode": arrivals, "l2_atomic_rtt_ns": round(rtt, 1),
                "latency_floor_ns": round(arrivals / rate * 1e9 + 2 * rtt, 1)}

    line = {"metric": "ns per grid barrier", "value": round(ns, 2), "unit": "ns", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic", "config": dict(base_cfg, barrier=gsrb.VARIANT_NAMES[c.variant],
                                                 cluster=c.cluster, fanin_groups=c.fanin_groups),
            "phase_only_ms": round(t_phase, 5), "roofline": roofline, "clocks": clk,
            "gpu_launches": int(l1 - l0),
            "e2e": {"value": round(e2e_ns, 2), "unit": "ns", "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                    "note": "per-episode time of the whole step incl. H2D/D2H copies and the FMA phase"}}

    if not args.no_extras:
        extras = {}
        for name, v in (("ccg_grid_sync", gsrb.BAR_CCG), ("reference_gsrb_soft2", gsrb.BAR_SOFT2),
                        ("reference_gcpusrb_flat", gsrb.BAR_FLAT), ("atomic_tree", gsrb.BAR_TREE)):
            cc = gsrb.cfg(variant=v, ctas_per_sm=args.k, threads=256)
            try:
                tt = statistics.median(time_barrier(gsrb, ctx, cc, args.episodes, args.fma, 3, 1))
                extras[name] = round((tt - t_phase) * 1e6 / args.episodes, 2)
            except (gsrb.GsrbError, AssertionError) as e:
                extras[name] = f"failed: {e}"
        line["comparison_ns_per_barrier"] = extras
        if isinstance(extras.get("ccg_grid_sync"), float):
            line["speedup_vs_ccg"] = round(extras["ccg_grid_sync"] / ns, 3)
        orc = load_oracle()
        peak, src = hbm_peak()
        red = reduce_numbers(gsrb, ctx, orc)
        red["hbm_frac"] = round(red["GB_s"] / peak, 4)
        red["peak_source"] = src
        line["reduce_2e24"] = red
        if dist.rank == 0:
            line["cpu_baseline"] = cpu_barrier_baseline(orc)

    if dist.rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    dist.close()


if __name__ == "__main__":
    main()
