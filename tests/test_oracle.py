"""The oracle pinned against the reference's golden vectors and known answers (CPU)."""
import pathlib
import time

import numpy as np
import pytest

GOLD = pathlib.Path(__file__).resolve().parent / "golden"
INF = 2**31 - 1


def test_scan_matches_reference_cpu_sum_scan(orc):
    # golden outputs produced by the reference's own cpu_sum_scan (scan/main.cu:11-21)
    z = np.load(GOLD / "scan_u32_golden.npz")
    for k in ("ones_1000", "u15_4099", "wrap_777", "single"):
        a, ref = z[k + "_in"], z[k + "_out"]
        assert np.array_equal(orc.scan_u32(a), ref), k
        assert np.array_equal(orc.scan_u32(a, threads=4), ref), k


def test_scan_all_ones_golden(orc):
    # scan/main.cu:37-41 fills the input with ones: the exclusive prefix is i
    n = 100_003
    assert np.array_equal(orc.scan_u32(np.ones(n, np.uint32)), np.arange(n, dtype=np.uint32))


def test_reduce_all_ones_golden(orc):
    # Reduce/test_reduce.cu:14-17: all ones, correct sum = N
    for n in (1, 7, 1 << 20, 303_104):
        assert orc.sum_i32(np.ones(n, np.int32)) == n
        assert orc.sum_i32(np.ones(n, np.int32), threads=3) == n


def test_reduce_matches_numpy(orc):
    a = np.random.default_rng(1).integers(-2**31, 2**31 - 1, 50_000, dtype=np.int64).astype(np.int32)
    assert orc.sum_i32(a) == int(a.astype(np.int64).sum())


def test_scan_f32_reference_is_fp64(orc):
    a = np.random.default_rng(3).random(10_000, dtype=np.float32)
    ref = orc.scan_f32_f64(a)
    want = np.concatenate([[0.0], np.cumsum(a.astype(np.float64))[:-1]])
    assert np.allclose(ref, want, rtol=0, atol=1e-9)


def _tiny(gsrb):
    return gsrb.Graph.read_gr(GOLD / "tiny.gr")


def test_bfs_dijkstra_known_answers(gsrb, orc):
    g = _tiny(gsrb)
    # hand-computed: BFS hops from 0 and Dijkstra distances of the classic 6-node example
    assert orc.bfs(g, 0).tolist() == [0, 1, 1, 2, 2, 1]
    assert orc.dijkstra(g, 0).tolist() == [0, 7, 9, 20, 20, 11]
    assert orc.traversed_edges(g, orc.bfs(g, 0)) == g.nedges


def test_bfs_unreachable_is_inf(gsrb, orc):
    g = gsrb.csr_from_edges(5, [0, 1], [1, 2])  # vertices 3, 4 isolated
    lv = orc.bfs(g, 0)
    assert lv.tolist() == [0, 1, 2, INF, INF]
    assert orc.traversed_edges(g, lv) == 4


def test_pagerank_fixed_point_two_cycle(gsrb, orc):
    # symmetric 2-vertex graph: x = (1-a) + a*x -> x = 1 after convergence
    g = gsrb.csr_from_edges(2, [0], [1])
    x = orc.pagerank(g, 0.85, 200)
    assert np.allclose(x, [1.0, 1.0], atol=1e-12)
    # 50 iterations from 1-a: x_k = 1 - a^(k+1)
    x50 = orc.pagerank(g, 0.85, 50)
    assert np.allclose(x50, 1 - 0.85**51, atol=1e-12)


def test_heterosync_golden_barrier_hand_case(orc):
    # Heterosync/main.cu:41-59 + :2993-3011 for a barrier kernel (syncPrim 37),
    # 1 ld/st, 2 TBs of 32 threads, 1 iteration: within every 32-word region
    # the second cache line (words 16..31) takes the first line's values.
    s = orc.heterosync_golden(37, 1, 2, 1, 1, 148, 32)
    assert s.size == 128
    want = np.arange(128, dtype=np.float32)
    for k in range(128):
        if k % 32 >= 16:
            want[k] = k - 16
    assert np.array_equal(s, want)
    # more iterations and repeats leave it unchanged (the copy is idempotent)
    assert np.array_equal(orc.heterosync_golden(37, 1, 2, 5, 10, 148, 32), want)


def test_heterosync_storage_sizes(orc):
    # Heterosync/main.cu:2561-2583
    assert orc.heterosync_storage_locs(37, 2, 296, 148, 32) == 296 * 32 * 3
    assert orc.heterosync_storage_locs(4, 2, 296, 148, 32) == 32 * 3
    assert orc.heterosync_storage_locs(16, 2, 296, 148, 32) == 2 * 32 * 3
    assert orc.heterosync_storage_locs(20, 2, 296, 148, 32) == 148 * 32 * 3


def test_cpu_barrier_model_no_stale_reads(orc):
    for nt, ng in ((4, 0), (6, 2), (8, 3)):
        ns, stale = orc.cpu_srb_barrier(nt, ng, 2000)
        assert stale == 0 and ns > 0


@pytest.mark.parametrize("nt,ng", [(5, 0), (8, 3), (12, 4)])
def test_cpu_barrier_model_injected_stalls(orc, nt, ng):
    # late arrivals and a completer stalled between its counter reset and its
    # publish: no participant may run ahead into the next episode
    ns, stale, stalls = orc.cpu_srb_barrier_stalls(nt, ng, 300, 40, nt * 31 + ng)
    assert stale == 0 and stalls > 0


@pytest.mark.parametrize("nt,ng,kill", [(4, 0, 2), (8, 3, 0), (8, 3, 7)])
def test_cpu_barrier_model_killed_participant_times_out(orc, nt, ng, kill):
    # a participant leaves for good after 50 episodes: the others' bounded
    # waits run out, the abort flag ends every wait, the run returns
    t0 = time.time()
    stale, timeouts = orc.cpu_srb_barrier_kill(nt, ng, 400, kill, 50, 200)
    assert timeouts >= 1 and stale == 0
    assert time.time() - t0 < 20
    # nobody killed: no timeouts
    stale, timeouts = orc.cpu_srb_barrier_kill(nt, ng, 200, -1, 0, 2000)
    assert timeouts == 0 and stale == 0


@pytest.mark.parametrize("nt,nctas,ng", [(4, 1184, 148), (8, 296, 148), (3, 10, 0), (16, 1184, 148)])
def test_cpu_barrier_model_many_ctas_per_thread(orc, nt, nctas, ng):
    # host threads carrying many participants each (the grid's CTAs)
    ns, stale = orc.cpu_srb_barrier_vcta(nt, nctas, ng, 300)
    assert stale == 0 and ns > 0


def test_cpu_semaphore_model_injected_stalls(orc):
    rate, W, R, mr, viol, stalls = orc.cpu_semaphore_stalls(8, 3, 4, 150, 8, 60, 2022)
    writers = sum(1 for t in range(8) if t % 4 == 0)
    assert W == writers * 150 * 8 and R == (8 - writers) * 150 * 8
    assert viol == 0 and 1 <= mr <= 3 and stalls > 0


def test_cpu_semaphore_model_exact_counts(orc):
    rate, W, R, mr, viol = orc.cpu_semaphore(6, 2, 3, 200, 10)
    writers = sum(1 for t in range(6) if t % 3 == 0)
    assert W == writers * 200 * 10
    assert R == (6 - writers) * 200 * 10
    assert viol == 0 and 1 <= mr <= 2
