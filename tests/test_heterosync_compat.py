"""A Heterosync-style program built only against the drop-in cudaLocks API
(bin/heterosync_compat, source tpds22-artifact_b200/apps/heterosync_compat.cu):
every barrier, mutex and priority-semaphore case must check out on the GPU."""
import pathlib
import subprocess

import pytest

BIN = pathlib.Path(__file__).resolve().parents[1] / "tpds22-artifact_b200" / "bin" / "heterosync_compat"
CASES = ["joinBarrier_helperSRB", "joinBarrier_helperNaiveSRB", "joinBarrier_helper", "joinLFBarrier_helper",
         "cudaMutexSpinLock", "cudaMutexEBOLock", "cudaMutexFALock", "cudaMutexSleepLock",
         "cudaSemaphoreSpinWaitPriority"]


def test_compat_program_built():
    assert BIN.exists()


@pytest.mark.gpu
def test_compat_program_passes(ctx):
    p = subprocess.run([str(BIN)], capture_output=True, text=True, timeout=600)
    lines = p.stdout.splitlines()
    assert p.returncode == 0, p.stdout + p.stderr
    for name in CASES:
        assert any(ln.startswith("PASS " + name) for ln in lines), (name, p.stdout)
    assert not any(ln.startswith("FAIL") for ln in lines)
