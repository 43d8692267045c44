import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


def _ensure_built():
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
    need = [os.path.join(ROOT, "readdygpu_b200", f) for f in ("libreaddy_b200.so", "libreaddy_workloads.so")]
    if not all(os.path.exists(p) for p in need):
        subprocess.check_call([sys.executable, os.path.join(ROOT, "readdygpu_b200", "build.py")], cwd=ROOT)


_ensure_built()


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    return O
