"""Host-side logic on CPU: configuration defaults, the policy's labels and
features, the autotuner's candidate sets, and bench.py's reference arm and
multi-process (gloo) path."""
import ctypes as C
import importlib.util
import json
import math
import os
import pathlib
import subprocess
import sys

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
PKG = ROOT / "tpds22-artifact_b200"


def _mod(name, path):
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, path)
    m = importlib.util.module_from_spec(spec)
    sys.modules[name] = m
    spec.loader.exec_module(m)
    return m


@pytest.fixture(scope="module")
def pol(gsrb):
    return _mod("gsrb_policy", PKG / "policy.py")


@pytest.fixture(scope="module")
def tune(gsrb):
    return _mod("gsrb_autotune", PKG / "autotune.py")


def test_cfg_default_matches_header(gsrb):
    c = gsrb.Cfg()
    gsrb.lib().gsrb_cfg_default(C.byref(c))
    assert c.variant == gsrb.BAR_CLUSTER and c.cluster == 2 and c.ctas_per_sm == 2 and c.threads == 256
    assert c.timeout_ms == 2000 and c.launch_mode == 1 and c.tile == 0
    # every variant has a name; the status strings are defined for every code
    for v in range(13):
        assert v in gsrb.VARIANT_NAMES
    for st in range(0, -11, -1):
        s = gsrb.lib().gsrb_status_string(st)
        assert s and b"unknown" not in s.lower()


def test_policy_weight_is_cost_sensitive(pol):
    assert pol._weight(100.0, 100.0) == pytest.approx(0.05)        # a tie hardly counts
    assert pol._weight(1000.0, 100.0) == pytest.approx(math.log2(10))
    assert pol._weight(100.0, 1000.0) == pytest.approx(math.log2(10))
    assert pol._weight(1e6, 1.0) == 4.0                              # clipped


def test_policy_level_times(pol):
    tr = np.zeros(4, dtype=[("t_ns", "<u8")])
    tr["t_ns"] = [100, 250, 600, 700]
    d = pol.level_times(tr)
    assert d[:3].tolist() == [150.0, 350.0, 100.0] and math.isnan(d[3])


def test_level_features_host_twin(gsrb):
    # the device evaluates the same function; check it against a restatement
    n, m, lvl, nf, mf, nu, mu, pnf, pdir = 4096, 65536, 3, 100, 1600, 3000, 40000, 10, 1
    f = gsrb.level_features(n, m, lvl, nf, mf, nu, mu, pnf, pdir)
    want = [math.log2(1 + nf), math.log2(1 + mf), math.log2(1 + nu), math.log2(1 + mu), nf / n, mf / (mu + 1),
            math.log2(1 + mf / nf), math.log2(1 + lvl), pdir, math.log2(n), math.log2(1 + m) - math.log2(n),
            math.log2(1 + nf) - math.log2(1 + pnf)]
    assert np.allclose(f, want, rtol=1e-5, atol=1e-6)


def test_mlp_init_layout(gsrb):
    p = gsrb.mlp_init(3)
    assert p.size == gsrb.mlp_param_count() == 32 * 12 + 32 + 32 * 32 + 32 + 4 * 32 + 4
    assert np.array_equal(p, gsrb.mlp_init(3)) and not np.array_equal(p, gsrb.mlp_init(4))
    assert np.all(np.isfinite(p))


def test_autotune_candidates_and_cfg_roundtrip(gsrb, tune):
    cands = tune.barrier_candidates(8)
    variants = {c["variant"] for c in cands}
    assert {gsrb.BAR_CCG, gsrb.BAR_FLAT, gsrb.BAR_FLIP, gsrb.BAR_FANOUT, gsrb.BAR_HIER} <= variants
    e = dict(variant=gsrb.BAR_FANOUT, wake_lines=2, spin_ns=64, ctas_per_sm=8, threads=256, bogus=1)
    c = tune.cfg_from(e)
    assert (c.variant, c.wake_lines, c.spin_ns, c.ctas_per_sm, c.threads) == (9, 2, 64, 8, 256)
    p = tune.CACHE.parent / "_tuned_test.json"
    try:
        tune.save_cache({"x": e}, p)
        assert tune.load_cache(p)["x"]["wake_lines"] == 2
    finally:
        if p.exists():
            p.unlink()
    assert tune.load_cache(ROOT / "does-not-exist.json") == {}
    # segment calls: only the protocols whose state does not depend on the team size
    for kind in ("reduce", "scan"):
        sc = tune.segment_candidates(kind)
        assert {c["variant"] for c in sc} == {gsrb.BAR_FANOUT, gsrb.BAR_FLIP, gsrb.BAR_FLAT}
        assert all(c["ctas_per_sm"] * c["threads"] <= 2048 for c in sc)
    assert {c["tile"] for c in tune.segment_candidates("reduce")} == {0}
    # the scan's register-resident candidates: fan-out, two groups, a chunk of
    # threads x 4 x (16 vectors a lane at <= 512 threads an SM, else 8) / 2
    reg = [c for c in tune.segment_candidates("scan") if c.get("form") == gsrb.FORM_REG]
    assert reg and all(c["variant"] == gsrb.BAR_FANOUT for c in reg)
    for c in reg:
        per = c["threads"] * (16 if c["ctas_per_sm"] * c["threads"] <= 512 else 8) * 4
        assert c["tile"] * 2 == per
    # the reduce tuner's chained candidates exist only on request and never for grid.sync
    assert not any(c.get("overlap") for c in tune.reduce_candidates(2, 256))
    chained = [c for c in tune.reduce_candidates(2, 256, overlap=True) if c.get("overlap")]
    assert chained and all(c["variant"] != gsrb.BAR_CCG for c in chained)


def test_bench_tail_summary_fits_the_tail():
    # the JSON line ends with one compact summary of every configuration, so a
    # reader that keeps only the last 1500 characters still sees them all
    import json
    bench = _mod("bench_under_test", ROOT / "bench.py")
    cf = {"C1_reduce_2e24": {"us": 9.68, "hbm_frac": 1.06, "unchained_hbm_frac": 0.66, "single_launch_cold_us": 20.5,
                             "bit_exact": True, "cpu_mt_GB_s": 57.2},
          "C2_barrier_k8": {f"F{f}": {"x_ccg": 1.1} for f in (0, 64, 1024)},
          "C2_barrier_reference_programs": {"k8": {"gsrb_ns": 24144.4, "gcpusrb_ns": 21390.7, "ccg_ns": 4188.8,
                                                   "atomic_tree_ns": 43595.4, "native_fanout_ns": 2237.0,
                                                   "native_flip_ns": 3299.3}},
          "C2_semaphore": {f"S{k}": {"acq_per_s": 123456.7} for k in (1, 2, 10, 120)},
          "C3_scan_2e28": {"u32_hbm_frac": 0.775, "f32_hbm_frac": 0.755, "u32_bit_exact": True, "cpu_mt_GB_s": 35.1},
          "C4_rmat22": {"bfs_learned_GTEPS": 271.1, "bfs_learned_vs_plain": 7.8, "sssp_GTEPS": 19.8,
                        "pr_frac_of_gather_floor": 0.613, "bfs_bit_exact": True, "sssp_bit_exact": True},
          "C4_grid2048": {"bfs_heuristic_ms": 29.8, "sssp_ms": 60.5},
          "C5_batch64": {"bfs_learned_vs_plain": 46.8, "bfs_learned_vs_heuristic": 1.04, "sssp_speedup": 4.1,
                         "bit_exact": True},
          "C5_segments64": {"reduce_hbm_frac": 0.648, "scan_hbm_frac": 0.555}}
    t = bench.tail_summary(cf)
    assert set(t) >= {"C1_reduce", "C2_barrier_k8_x_ccg", "C3_scan", "C4_rmat22", "C5_batch64",
                      "C5_segments64_hbm_frac"}
    assert t["C1_reduce"]["hbm_frac"] == 1.06 and t["C4_rmat22"]["exact"] is True
    assert len(json.dumps({"summary": t})) < 1400


def _bench_env():
    env = dict(os.environ)
    env["MASTER_ADDR"] = "127.0.0.1"
    return env


def test_bench_reference_arm_line():
    p = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], capture_output=True, text=True, timeout=600, env=_bench_env())
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["higher_is_better"] is False and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["value"] == d["value"]


def test_bench_two_ranks_gloo():
    # torchrun with two CPU ranks: rank 0 alone prints the reference line, rank 1 exits cleanly
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", "29633", str(ROOT / "bench.py"), "--impl",
           "reference", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=900, env=_bench_env())
    assert p.returncode == 0, p.stderr[-3000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    assert json.loads(lines[0])["n_gpus"] == 2


def _max_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    bench = _mod("bench_under_test", ROOT / "bench.py")
    d = bench.Dist()
    v = d.max(float(10 * (rank + 1)))
    d.barrier()
    d.close()
    q.put((rank, v))


def test_dist_max_over_ranks_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_max_worker, args=(r, 2, 29655, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = dict(q.get(timeout=300) for _ in ps)
    for p in ps:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert got == {0: 20.0, 1: 20.0}


def _fake_trace(gsrb, nfs, mfs):
    tr = np.zeros(len(nfs), dtype=gsrb.TRACE_DTYPE)
    tr["level"] = np.arange(1, len(nfs) + 1)
    tr["nf"] = nfs
    tr["mf"] = mfs
    tr["nu"] = 1000 - np.cumsum(nfs)
    tr["mu"] = 16000 - np.cumsum(mfs)
    tr["t_ns"] = np.cumsum([0] + [100] * (len(nfs) - 1))
    return tr


def test_trace_files_roundtrip_and_labels(gsrb, pol, tmp_path):
    push = _fake_trace(gsrb, [1, 10, 300, 50], [16, 160, 4800, 800])
    rec = {"n": 1000, "m": 16000, "src": 0, "push": push, "pull": push.copy(), "topo": push.copy(),
           "push_ns": np.array([100.0, 900.0, 4000.0, np.nan]),
           "pull_ns": np.array([5000.0, 1000.0, 400.0, np.nan]),
           "topo_ns": np.array([300.0, 900.0, 8000.0, np.nan])}
    path = tmp_path / "traces.npz"
    pol.save_traces(path, [rec, rec])
    back = pol.load_traces(path)
    assert len(back) == 2 and back[1]["n"] == 1000 and np.array_equal(back[0]["push"], push)
    X, Y, M = pol.dataset(back)
    assert X.shape == (8, 12) and Y.shape == (8, 4)
    # level 1 (index 0): no pull label (the first level is always a push)
    assert M[0, 0] == 0.0
    # level 3: pull 10x faster -> label 1, weight log2(10)
    assert Y[2, 0] == 1.0 and M[2, 0] == pytest.approx(math.log2(10))
    # level 2: pull 1.1x slower -> label 0, small weight
    assert Y[1, 0] == 0.0 and M[1, 0] < 0.2
    # next-frontier regression target
    assert Y[0, 2] == pytest.approx(math.log2(11)) and Y[3, 2] == 0.0


def test_level_rows_capped_per_graph(gsrb, pol):
    # a long traversal (a mesh) weighs as much as LEVEL_CAP levels in total
    L = 4 * pol.LEVEL_CAP
    nfs = [1] + [2] * (L - 1)
    push = _fake_trace(gsrb, nfs, [4] * L)
    t = np.full(L, 100.0)
    rec = {"n": 100000, "m": 400000, "src": 0, "push": push, "pull": push.copy(), "topo": push.copy(),
           "push_ns": t, "pull_ns": t * 2, "topo_ns": t * 2}
    X, Y, M = pol.features_labels(rec)
    assert X.shape == (L, 12)
    assert M[:, 2].sum() == pytest.approx(pol.LEVEL_CAP)
    short = _fake_trace(gsrb, [1, 10, 300, 50], [16, 160, 4800, 800])
    rec2 = dict(rec, push=short, pull=short.copy(), topo=short.copy(), push_ns=t[:4], pull_ns=t[:4] * 2,
                topo_ns=t[:4] * 2)
    _, _, M2 = pol.features_labels(rec2)
    assert M2[:, 2].sum() == 4.0


def test_launch_label_first_level_only(gsrb, pol, tmp_path):
    push = _fake_trace(gsrb, [1, 10, 300, 50], [16, 160, 4800, 800])
    rec = {"n": 1000, "m": 16000, "src": 0, "push": push, "pull": push.copy(), "topo": push.copy(),
           "push_ns": np.array([100.0, 900.0, 4000.0, np.nan]),
           "pull_ns": np.array([5000.0, 1000.0, 400.0, np.nan]),
           "topo_ns": np.array([300.0, 900.0, 8000.0, np.nan]),
           "launch_ms": np.array([2.0, 0.5])}
    path = tmp_path / "traces.npz"
    pol.save_traces(path, [rec])
    back = pol.load_traces(path)
    assert np.array_equal(back[0]["launch_ms"], [2.0, 0.5])
    X, Y, M = pol.dataset(back)
    # no sampled sources: one launch row, the first level's features, after the 4 level rows
    assert X.shape == (5, 12) and not M[:4, 3].any() and not M[4, :3].any()
    np.testing.assert_array_equal(X[4], gsrb.level_features(1000, 16000, 1, 1, 16, 999, 16000 - 16, 1, 0))
    np.testing.assert_array_equal(X[4], X[0])
    # configuration 1 is 4x faster: head 3 target log2(t0 / t1) = 2
    assert Y[4, 3] == pytest.approx(2.0) and M[4, 3] == pol.LAUNCH_WEIGHT
    # sampled sources: one row per source degree, all with the graph's label
    rec["launch_degs"] = np.array([16, 3, 40])
    pol.save_traces(path, [rec])
    X, Y, M = pol.dataset(pol.load_traces(path))
    assert X.shape == (7, 12) and np.all(Y[4:, 3] == Y[4, 3]) and np.all(M[4:, 3] == pol.LAUNCH_WEIGHT)
    np.testing.assert_array_equal(X[5], gsrb.level_features(1000, 16000, 1, 1, 3, 999, 16000 - 3, 1, 0))
    # the target is clipped to [-4, 4]
    rec["launch_ms"] = np.array([1.0, 1000.0])
    _, Y, _ = pol.features_labels(rec)
    assert np.all(Y[4:, 3] == -4.0)
    # traces without launch times carry no launch rows
    del rec["launch_ms"]
    X, _, M = pol.features_labels(rec)
    assert X.shape == (4, 12) and not M[:, 3].any()


def test_segments_layout(gsrb):
    # every segment gets at least one CTA, the rest go in proportion to length,
    # the teams tile the grid in order
    rng = np.random.default_rng(1)
    for k, grid in ((1, 296), (5, 5), (64, 296), (127, 296), (127, 1184)):
        lens = rng.integers(0, 1 << 20, k)
        lens[::7] = 0
        off = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
        first, count = gsrb.segments_layout(off, grid)
        assert first[0] == 0 and np.all(count >= 1) and int(count.sum()) == grid
        assert np.array_equal(first[1:], first[:-1] + count[:-1])
        if lens.sum():
            extra = count.astype(np.int64) - 1
            share = (grid - k) * lens / lens.sum()
            assert np.all(np.abs(extra - share) <= 1.0 + 1e-9)
    # no elements at all: one CTA each, the last segment the rest
    first, count = gsrb.segments_layout(np.zeros(4, np.uint64), 10)
    assert count.tolist() == [1, 1, 8]
    with pytest.raises(gsrb.GsrbError):
        gsrb.segments_layout(np.arange(6, dtype=np.uint64), 4)  # grid < k


def test_sssp_labels(pol):
    # widths within 3 % of the faster configuration's best are averaged in
    # log2(width / mean weight); the launch label is the clipped log-ratio
    t = np.array([[9.0, 5.0, 4.0, 4.1, 4.0, 6.0],
                  [20.0, 10.0, 8.0, 8.0, 8.0, 8.0]])
    y2, y3 = pol.sssp_labels(t, 128.0)
    want = np.mean([np.log2(d / 128.0) for d in (1024, 4096, 16384)])
    assert abs(y2 - want) < 1e-9
    assert abs(y3 - np.log2(4.0 / 8.0)) < 1e-9
    y2, y3 = pol.sssp_labels(np.array([[100.0] * 6, [1.0] * 6]), 1.0)
    assert y3 == 4.0  # clipped


def test_sssp_features_host(gsrb):
    f = np.zeros(12, np.float32)
    gsrb.lib().gsrb_sssp_features(1 << 20, 16 << 20, 5000, 7, 128.0, 1, 255, 1, f.ctypes.data)
    assert abs(f[0] - 20.0) < 1e-5 and abs(f[2] - np.log2(17.0)) < 1e-5
    assert abs(f[4] - 3.0) < 1e-5 and f[8] == 1.0
    assert abs(f[11] - (f[0] - 2 * f[2])) < 1e-5


def test_bench_tuning_note_keeps_grid_sync_beside(gsrb):
    # the graphs' launch tuning reports the library's own pick and grid.sync's
    # best shape beside it, from the tuner's sorted table
    bench = _mod("bench_under_test", ROOT / "bench.py")
    table = [(26.5, dict(variant=gsrb.BAR_CCG, ctas_per_sm=1, threads=256)),
             (27.3, dict(variant=gsrb.BAR_FLIP, fanin_groups=1, ctas_per_sm=1, threads=256)),
             (30.4, dict(variant=gsrb.BAR_FLIP, fanin_groups=1, ctas_per_sm=2, threads=256))]
    note = bench._tuning_note(gsrb, table[1][1], table)
    assert note["cfg"]["variant"] == gsrb.BAR_FLIP and note["tuning_ms"] == 27.3
    assert note["grid_sync_best_ms"] == 26.5 and note["grid_sync_best_cfg"]["ctas_per_sm"] == 1
