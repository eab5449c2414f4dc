"""The Heterosync microbenchmark program (bin/allSyncPrims-1kernel, source
tpds22-artifact_b200/apps/allSyncPrims.cu) against the oracle's restatement of
the harness's golden replay (Heterosync/main.cu:41-59, 2987-3146).

Every shift of a column is the same copy, so the storage array records how many
times each column was shifted (up to NUM_LDST, where the column saturates).  The
cases keep the number of shifts per column below NUM_LDST so that a lost,
doubled or torn critical section changes the result."""
import pathlib
import re
import subprocess

import numpy as np
import pytest

BIN = pathlib.Path(__file__).resolve().parents[1] / "tpds22-artifact_b200" / "bin" / "allSyncPrims-1kernel"
TPB = 32

BARRIERS = {
    0: "atomicTreeBarrUniq", 1: "atomicTreeBarrUniqLocalExch", 2: "lfTreeBarrUniq", 3: "lfTreeBarrUniqLocalExch",
    37: "atomicTreeBarrUniqSRB", 38: "atomicTreeBarrUniqLocalExchSRB", 39: "atomicTreeBarrUniqNaiveSRB",
    40: "atomicTreeBarrUniqLocalExchNaiveSRB", 41: "atomicTreeBarrUniqNaiveAllSRB",
    42: "atomicTreeBarrUniqLocalExchNaiveAllSRB", 43: "atomicTreeBarrUniqHybridSRB",
    44: "atomicTreeBarrUniqLocalExchHybridSRB", 45: "atomicTreeBarrUniqCCG", 46: "atomicTreeBarrUniqLocalExchCCG"}
MUTEXES = {4: "spinMutex", 5: "spinMutexEBO", 6: "sleepMutex", 7: "faMutex"}
UNIQ_MUTEXES = {20: "spinMutexUniq", 21: "spinMutexEBOUniq", 22: "sleepMutexUniq", 23: "faMutexUniq"}
SEMAPHORES = {8: "spinSem1", 9: "spinSem2", 10: "spinSem10", 11: "spinSem120", 12: "spinSemEBO1",
              13: "spinSemEBO2", 14: "spinSemEBO10", 15: "spinSemEBO120", 16: "PRspinSem1", 17: "PRspinSem2",
              18: "PRspinSem10", 19: "PRspinSem120", 32: "PRspinSemEBO1", 33: "PRspinSemEBO2",
              34: "PRspinSemEBO10", 35: "PRspinSemEBO120"}
UNIQ_SEMAPHORES = {24: "spinSemUniq1", 25: "spinSemUniq2", 26: "spinSemUniq10", 27: "spinSemUniq120",
                   28: "spinSemEBOUniq1", 29: "spinSemEBOUniq2", 30: "spinSemEBOUniq10", 31: "spinSemEBOUniq120"}


def _run(args, tmp_path, timeout=300):
    out = tmp_path / "storage.bin"
    p = subprocess.run([str(BIN), *map(str, args), "-o", str(out)], capture_output=True, text=True, timeout=timeout)
    return p, out


def _check(orc, tmp_path, prim, name, ldst, ntbs, iters, repeats):
    p, out = _run([name, ldst, ntbs, iters, "-r", repeats], tmp_path)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    assert "PASSED!" in p.stdout
    nsm = int(re.search(r"# SM: (\d+)", p.stdout).group(1))
    got = np.fromfile(out, dtype=np.float32)
    want = orc.heterosync_golden(prim, ldst, ntbs, iters, repeats, nsm, TPB)
    assert got.shape == want.shape
    bad = np.flatnonzero(got != want)
    assert bad.size == 0, (name, bad[:10], got[bad[:10]], want[bad[:10]])
    return p.stdout, nsm


@pytest.fixture(scope="module")
def nsm():
    import torch
    return torch.cuda.get_device_properties(0).multi_processor_count


def test_program_built():
    assert BIN.exists()


def test_unknown_primitive_and_usage():
    # both are rejected before any CUDA call, so this runs without a GPU
    p = subprocess.run([str(BIN), "noSuchPrim", "1", "1", "1"], capture_output=True, text=True, timeout=60)
    assert p.returncode != 0 and "Unknown synchronization primitive" in p.stderr
    p = subprocess.run([str(BIN)], capture_output=True, text=True, timeout=60)
    assert p.returncode != 0 and "usage" in p.stderr and "atomicTreeBarrUniqLocalExchCCG" in p.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("prim", sorted(BARRIERS))
def test_barrier_kernels_two_ctas_per_sm(orc, tmp_path, ctx, nsm, prim):
    # 3 iterations x 2 launches: 6 shifts per column (12 with the local exchange) < 24
    out, _ = _check(orc, tmp_path, prim, BARRIERS[prim], 24, 2 * nsm, 3, 2)
    assert re.search(r"elapsed time: [0-9.]+ ms, average: [0-9.]+ ms", out)


@pytest.mark.gpu
@pytest.mark.parametrize("prim", [2, 3, 37, 38, 43, 44, 45])
def test_barrier_kernels_eight_ctas_per_sm(orc, tmp_path, ctx, nsm, prim):
    # the hybrid switches from the library barrier to the tree SRB at 8 CTAs per SM
    _check(orc, tmp_path, prim, BARRIERS[prim], 16, 8 * nsm, 2, 2)


@pytest.mark.gpu
@pytest.mark.parametrize("prim", [0, 37, 39, 45])
def test_barrier_kernels_fewer_ctas_than_sms(orc, tmp_path, ctx, nsm, prim):
    _check(orc, tmp_path, prim, BARRIERS[prim], 16, nsm // 2 + 3, 4, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("prim", sorted(MUTEXES))
def test_mutex_kernels_exact_shift_count(orc, tmp_path, ctx, prim):
    # 24 CTAs, one critical section each: 24 shifts of the one shared column block < 32
    _check(orc, tmp_path, prim, MUTEXES[prim], 32, 24, 1, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("prim", sorted(MUTEXES))
def test_mutex_kernels_contended(orc, tmp_path, ctx, nsm, prim):
    _check(orc, tmp_path, prim, MUTEXES[prim], 8, 2 * nsm, 3, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("prim", sorted(UNIQ_MUTEXES))
def test_uniq_mutex_kernels(orc, tmp_path, ctx, nsm, prim):
    # 4 CTAs per group x 2 iterations: 8 shifts of each group's columns < 16
    _check(orc, tmp_path, prim, UNIQ_MUTEXES[prim], 16, 4 * nsm, 2, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("prim", sorted(SEMAPHORES))
def test_semaphore_writers_exact_shift_count(orc, tmp_path, ctx, prim):
    # fewer CTAs than SMs: every CTA is its group's writer and shifts the same
    # columns, so writers must exclude each other: 8 x 2 = 16 shifts < 32
    _check(orc, tmp_path, prim, SEMAPHORES[prim], 32, 8, 2, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("prim", sorted(SEMAPHORES))
def test_semaphore_readers_and_writers(orc, tmp_path, ctx, nsm, prim):
    _check(orc, tmp_path, prim, SEMAPHORES[prim], 8, 2 * nsm, 2, 1)


@pytest.mark.gpu
@pytest.mark.parametrize("prim", sorted(UNIQ_SEMAPHORES))
def test_uniq_semaphore_kernels(orc, tmp_path, ctx, nsm, prim):
    # one writer per group shifts each of the group's columns once per iteration: 6 < 16
    _check(orc, tmp_path, prim, UNIQ_SEMAPHORES[prim], 16, 4 * nsm, 3, 2)


@pytest.mark.gpu
def test_local_exchange_needs_equal_groups(tmp_path, ctx, nsm):
    p, _ = _run(["atomicTreeBarrUniqLocalExchSRB", 4, 2 * nsm + 1, 1], tmp_path)
    assert p.returncode != 0 and "multiple of" in p.stderr


@pytest.mark.gpu
def test_banner_lines_match_the_reference(orc, tmp_path, ctx):
    # Heterosync/main.cu:2670,2702,2734 print size 2 for the size-120 spin semaphores
    out, _ = _check(orc, tmp_path, 11, "spinSem120", 8, 8, 1, 1)
    assert "\nspin_lock_sem_002_001\n" in out
    out, _ = _check(orc, tmp_path, 37, "atomicTreeBarrUniqSRB", 8, 8, 1, 1)
    assert "\natomic_tree_barrier_SRB_001\n" in out
