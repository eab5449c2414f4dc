"""Policy MLP kernels: forward and gradients against the FP64 oracle, training."""
import ctypes as C
import pathlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = pathlib.Path(__file__).resolve().parents[1]
GRAD_REL_TOL = 1e-4


def _orc():
    lib = C.CDLL(str(ROOT / "oracle" / "lib" / "liboracle.so"))
    lib.orc_mlp_loss_grad.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_void_p, C.c_void_p]
    lib.orc_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    return lib


def _data(B, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(B, 12)).astype(np.float32)
    Y = np.concatenate([rng.integers(0, 2, (B, 2)), rng.normal(size=(B, 2))], axis=1).astype(np.float32)
    M = np.ones((B, 4), np.float32)
    M[:, 3] = 0
    return X, Y, M


def test_mlp_forward_matches_oracle(gsrb, ctx):
    lib = _orc()
    p = gsrb.mlp_init(1)
    X, _, _ = _data(300)
    got = gsrb.mlp_forward(ctx, p, X)
    ref = np.zeros((300, 4), np.float64)
    lib.orc_mlp_forward(p.ctypes.data, X.ctypes.data, 300, ref.ctypes.data)
    assert np.max(np.abs(got - ref)) <= 1e-4 * max(1.0, np.max(np.abs(ref)))


def test_mlp_gradient_matches_oracle(gsrb, ctx):
    lib = _orc()
    p = gsrb.mlp_init(2)
    X, Y, M = _data(777, seed=3)
    g, loss = gsrb.mlp_loss_grad(ctx, p, X, Y, M)
    gref = np.zeros(p.size, np.float64)
    L = C.c_double()
    lib.orc_mlp_loss_grad(p.ctypes.data, X.ctypes.data, Y.ctypes.data, M.ctypes.data, 777, gref.ctypes.data,
                          C.byref(L))
    assert abs(loss - L.value) <= GRAD_REL_TOL * max(1.0, abs(L.value))
    scale = max(np.max(np.abs(gref)), 1e-6)
    assert np.max(np.abs(g - gref)) <= GRAD_REL_TOL * scale


def test_mlp_training_reduces_loss(gsrb, ctx):
    # a learnable rule: head 0 = (x0 + x1 > 0), head 2 = 2*x2 - x3
    rng = np.random.default_rng(7)
    X = rng.normal(size=(2048, 12)).astype(np.float32)
    Y = np.zeros((2048, 4), np.float32)
    Y[:, 0] = (X[:, 0] + X[:, 1] > 0)
    Y[:, 2] = 2 * X[:, 2] - X[:, 3]
    M = np.zeros((2048, 4), np.float32)
    M[:, 0] = 1
    M[:, 2] = 1
    p0 = gsrb.mlp_init(11)
    p, hist = gsrb.mlp_train(ctx, p0, X, Y, M, steps=600, lr=3e-3)
    assert hist[-1] < 0.25 * hist[0]
    out = gsrb.mlp_forward(ctx, p, X)
    acc = np.mean((out[:, 0] > 0) == (Y[:, 0] > 0.5))
    assert acc > 0.95
    # deterministic: the same run gives the same parameters
    p2, _ = gsrb.mlp_train(ctx, p0, X, Y, M, steps=600, lr=3e-3)
    assert np.array_equal(p, p2)
