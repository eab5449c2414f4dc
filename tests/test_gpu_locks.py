"""Mutexes and semaphores on the GPU: exact final counters, exclusion and capacity."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _counters(ctx):
    return ctx.array(8, np.uint32).zero()


@pytest.mark.parametrize("kind", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("cap", [1, 2, 10, 120])
def test_semaphore_counts_exact(gsrb, ctx, kind, cap):
    k, iters, incs, every = 2, 4, 100, 11
    c = gsrb.cfg(ctas_per_sm=k, threads=256, timeout_ms=3000)
    cnt = _counters(ctx)
    st = ctx.semaphore_bench(c, kind, cap, every, iters, incs, cnt)
    gsrb.check(st, "semaphore_bench")
    W, R, inside, maxr, viol, acq, tmo, _ = cnt.download().tolist()
    grid = k * ctx.num_sms
    writers = len([b for b in range(grid) if b % every == 0])
    assert tmo == 0 and viol == 0 and inside == 0
    assert acq == grid * iters
    assert W == writers * iters * incs          # plain RMW: any writer overlap would lose updates
    assert R == (grid - writers) * iters * incs
    assert 1 <= maxr <= cap


@pytest.mark.parametrize("kind", [1, 3])
@pytest.mark.parametrize("cap", [2, 10])
def test_semaphore_backoff_baselines_exact(gsrb, ctx, kind, cap):
    # The reference's backoff (EBO) semaphores with the reference's asymmetric
    # backoff (writers exponential, readers linear): every acquire completes,
    # counts are exact, no exclusion violation.  (With equal backoff for readers
    # and writers the readers kept the writers out for seconds.)
    k, iters, incs, every = 1, 4, 100, 11
    c = gsrb.cfg(ctas_per_sm=k, threads=256, timeout_ms=3000)
    cnt = _counters(ctx)
    gsrb.check(ctx.semaphore_bench(c, kind, cap, every, iters, incs, cnt), "semaphore_bench")
    W, R, inside, maxr, viol, acq, tmo, _ = cnt.download().tolist()
    grid = k * ctx.num_sms
    writers = len([b for b in range(grid) if b % every == 0])
    assert viol == 0 and tmo == 0 and inside == 0 and 1 <= maxr <= cap
    assert acq == grid * iters
    assert W == writers * iters * incs and R == (grid - writers) * iters * incs


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_mutex_counts_exact(gsrb, ctx, kind):
    k, iters, incs = 1, 3, 50
    c = gsrb.cfg(ctas_per_sm=k, threads=128, timeout_ms=3000)
    cnt = _counters(ctx)
    gsrb.check(ctx.mutex_bench(c, kind, iters, incs, cnt), "mutex_bench")
    W, R, inside, maxr, viol, acq, tmo, _ = cnt.download().tolist()
    grid = k * ctx.num_sms
    assert tmo == 0 and viol == 0
    assert acq == grid * iters and W == grid * iters * incs


def test_semaphore_full_residency(gsrb, ctx):
    # 148 x 8 CTAs of 256 threads contend on one priority semaphore
    c = gsrb.cfg(ctas_per_sm=8, threads=256, timeout_ms=5000)
    cnt = _counters(ctx)
    gsrb.check(ctx.semaphore_bench(c, gsrb.SEM_PRIORITY, 10, 11, 2, 100, cnt))
    W, R, inside, maxr, viol, acq, tmo, _ = cnt.download().tolist()
    grid = 8 * ctx.num_sms
    writers = len([b for b in range(grid) if b % 11 == 0])
    assert viol == 0 and tmo == 0 and W == writers * 200 and R == (grid - writers) * 200


@pytest.mark.parametrize("cap", [1, 2, 120])
def test_semaphore_overpost_detected(gsrb, ctx, cap):
    # a post without its wait pushes the count above its maximum: the next
    # waits report the invariant at once (no deadline), and the context and
    # a fresh semaphore work afterwards
    out = ctx.array(2, np.uint32).zero()
    assert ctx.semaphore_fault_overpost(cap, out) == gsrb.ERR_INVARIANT
    assert out.download().tolist() == [0, 0]
    assert ctx.status()[0] == 0
    cnt = _counters(ctx)
    gsrb.check(ctx.semaphore_bench(gsrb.cfg(ctas_per_sm=1, threads=64, timeout_ms=3000), 4, cap, 5, 2, 10, cnt))
    assert cnt.download().tolist()[6] == 0


@pytest.mark.parametrize("cap", [1, 10])
def test_semaphore_writer_timeout_hands_turn_on(gsrb, ctx, cap):
    # a writer that is served but gives up on the count (a reader slot is held
    # by its own CTA) reports LOCK_TIMEOUT and hands its turn on: the next
    # writer of the same record is served, and the record ends balanced
    out = ctx.array(5, np.uint32).zero()
    assert ctx.semaphore_fault_writer_timeout(cap, out) == gsrb.ERR_LOCK_TIMEOUT
    r, w1, w2, count, serving = out.download().tolist()
    assert (r, w1, w2) == (1, 0, 1)
    assert count == cap + 1 and serving == 2
    assert ctx.status()[0] == 0
