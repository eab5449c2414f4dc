"""Shared fixtures: the libgsrb binding, the CPU oracle, a GPU context."""
import importlib.util
import pathlib
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
PKG = ROOT / "tpds22-artifact_b200"
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device")
    config.addinivalue_line("markers", "slow: long-running (full-size) case")


def _load_binding():
    if "gsrb_b200" in sys.modules:
        return sys.modules["gsrb_b200"]
    spec = importlib.util.spec_from_file_location("gsrb_b200", PKG / "gsrb.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gsrb_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _ensure_built():
    lib = PKG / "lib" / "libgsrb.so"
    if not lib.exists() or not (PKG / "bin" / "bfs_gsrb").exists():
        subprocess.run(["make", "-C", str(PKG), "-j8"], check=True, capture_output=True)
    olib = ROOT / "oracle" / "lib" / "liboracle.so"
    if not olib.exists():
        subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True, capture_output=True)


_ensure_built()


@pytest.fixture(scope="session")
def gsrb():
    return _load_binding()


@pytest.fixture(scope="session")
def orc():
    import oracle_binding
    return oracle_binding


def _has_gpu():
    try:
        out = subprocess.run(["nvidia-smi", "-L"], capture_output=True, text=True, timeout=30)
        return out.returncode == 0 and "GPU" in out.stdout
    except Exception:
        return False


@pytest.fixture(scope="session")
def ctx(gsrb):
    if not _has_gpu():
        pytest.skip("no GPU")
    c = gsrb.Context(0)
    yield c
    c.close()
