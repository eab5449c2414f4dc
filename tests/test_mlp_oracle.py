"""The policy MLP's CPU oracle (FP64) against finite differences (CPU only)."""
import ctypes as C
import pathlib

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _orc_mlp():
    lib = C.CDLL(str(ROOT / "oracle" / "lib" / "liboracle.so"))
    lib.orc_mlp_loss_grad.argtypes = [C.c_void_p] * 4 + [C.c_int, C.c_void_p, C.c_void_p]
    lib.orc_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    return lib


def _loss_grad(lib, p, X, Y, M):
    g = np.zeros(p.size, np.float64)
    L = C.c_double()
    lib.orc_mlp_loss_grad(p.ctypes.data, X.ctypes.data, Y.ctypes.data, M.ctypes.data, X.shape[0], g.ctypes.data,
                          C.byref(L))
    return L.value, g


def test_mlp_oracle_gradient_matches_finite_differences(gsrb):
    lib = _orc_mlp()
    rng = np.random.default_rng(0)
    p = gsrb.mlp_init(5)
    B = 16
    X = rng.normal(size=(B, 12)).astype(np.float32)
    Y = np.concatenate([rng.integers(0, 2, (B, 2)), rng.normal(size=(B, 2))], axis=1).astype(np.float32)
    M = np.ones((B, 4), np.float32)
    M[::2, 3] = 0  # head 3 (the launch choice) is labelled on some rows only
    L, g = _loss_grad(lib, p, X, Y, M)
    def fd(i, eps):
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        return (_loss_grad(lib, pp, X, Y, M)[0] - _loss_grad(lib, pm, X, Y, M)[0]) / (2 * eps)

    idx = rng.choice(p.size, 80, replace=False)
    checked = 0
    for i in idx:
        a, b = fd(i, 2e-3), fd(i, 1e-3)
        if abs(a - b) > 1e-3 * max(1.0, abs(b)):
            continue  # the perturbation crossed a ReLU kink: finite differences are not valid here
        checked += 1
        assert abs(b - g[i]) <= 1e-3 * max(1.0, abs(g[i])) + 1e-5, (i, b, g[i])
    assert checked >= 60


def test_level_features_shape(gsrb):
    f = gsrb.level_features(1 << 20, 1 << 24, 3, 1000, 50_000, 900_000, 20_000_000, 10, 0)
    assert f.shape == (12,) and np.all(np.isfinite(f))
    assert abs(f[0] - np.log2(1001)) < 1e-5
