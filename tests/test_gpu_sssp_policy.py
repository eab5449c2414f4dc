"""The learned SSSP schedule: a policy network trained on timed SSSP runs of
training graphs picks, per traversal, the bucket width and the launch
configuration.  On held-out graphs its distances stay bit-exact (the schedule
never changes the arithmetic) and its time is compared with the reference's
fixed schedule (DELTA = 10000, LONESTAR/apps/sssp/support.cu:10, one launch
shape for every graph)."""
import importlib.util
import pathlib
import statistics

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = pathlib.Path(__file__).resolve().parents[1]
REFERENCE_DELTA = 10000
# learned total time over the held-out graphs may exceed the fixed schedule's by at most this
MARGIN = 1.10


def _policy():
    spec = importlib.util.spec_from_file_location("gsrb_policy", ROOT / "tpds22-artifact_b200" / "policy.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="module")
def trained(gsrb, ctx):
    pol = _policy()
    train = [gsrb.rmat(s, 16, seed=9000 + s) for s in (12, 13, 14, 15, 16)]
    train += [gsrb.grid2d(w, h, seed=9100 + w + h, wlo=1, whi=1000)
              for w, h in ((128, 128), (256, 64), (256, 256), (512, 128), (512, 512))]
    X, Y, M = [], [], []
    for g in train:
        dg = ctx.graph(g)
        x, y, m, _ = pol.sssp_collect(ctx, dg, reps=1)
        X.append(x)
        Y.append(y)
        M.append(m)
        dg.free()
    params, hist = pol.sssp_train(ctx, np.concatenate(X), np.concatenate(Y), np.concatenate(M), steps=2000)
    assert hist[-1] < hist[0]
    return params


def _median_ms(dg, out, delta, c, reps=5):
    ts = []
    for _ in range(reps):
        rc, st = dg.sssp(0, out, delta, c)
        assert rc == 0
        ts.append(st.kernel_ms)
    return statistics.median(ts), st


def test_learned_sssp_held_out(gsrb, ctx, orc, trained):
    pol = _policy()
    held = [gsrb.rmat(14, 16, seed=4242), gsrb.rmat(17, 16, seed=4343),
            gsrb.grid2d(384, 384, seed=4444, wlo=1, whi=1000), gsrb.grid2d(640, 160, seed=4545, wlo=1, whi=1000)]
    cands = pol.launch_candidates()
    t_learned = t_fixed = 0.0
    differs = False
    for g in held:
        dg = ctx.graph(g)
        dg.set_sssp_policy(trained)
        dg.set_launch_choices(*cands)
        delta, choice, _, _ = dg.sssp_plan(0)
        differs |= delta != REFERENCE_DELTA or choice != 0
        out = ctx.array(g.nnodes, np.int32)
        want = orc.dijkstra(g, 0)
        tl, st = _median_ms(dg, out, gsrb.SSSP_DELTA_LEARNED, None)
        assert st.delta == delta and st.launch == 1 + choice
        assert np.array_equal(out.download(), want)
        tf, _ = _median_ms(dg, out, REFERENCE_DELTA, cands[0])
        assert np.array_equal(out.download(), want)
        t_learned += tl
        t_fixed += tf
        dg.free()
    assert differs, "the policy reproduced the fixed schedule on every held-out graph"
    assert t_learned <= MARGIN * t_fixed, (t_learned, t_fixed)


def test_learned_sssp_batch_bit_exact(gsrb, ctx, orc, trained):
    graphs = [gsrb.rmat(s, 16, seed=5000 + s) for s in (12, 14, 15)] + [gsrb.grid2d(200, 100, seed=51)]
    dgs = [ctx.graph(g) for g in graphs]
    for dg in dgs:
        dg.set_sssp_policy(trained)
    outs = [ctx.array(g.nnodes, np.int32) for g in graphs]
    b = gsrb.Batch(ctx, dgs, gsrb.cfg(variant=gsrb.BAR_FANOUT, ctas_per_sm=2, threads=512, wake_lines=4))
    gsrb.check(b.sssp([0] * len(graphs), outs, gsrb.SSSP_DELTA_LEARNED), "batch sssp learned")
    rc, st = b.stats()
    gsrb.check(rc, "batch stats")
    for g, o in zip(graphs, outs):
        assert np.array_equal(o.download(), orc.dijkstra(g, 0))
    b.free()
    for dg in dgs:
        dg.free()


def test_sssp_plan_needs_a_policy(gsrb, ctx):
    g = gsrb.rmat(10, 8, seed=3)
    dg = ctx.graph(g)
    out = ctx.array(g.nnodes, np.int32)
    rc, _ = dg.sssp(0, out, gsrb.SSSP_DELTA_LEARNED)
    assert rc == gsrb.ERR_STATE
    dg.free()
