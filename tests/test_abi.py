"""The C-ABI libraries load and export every symbol their headers declare."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b((?:rdgpu|Java)_\w+)\s*\(", src)))


def test_engine_exports_every_declared_symbol():
    import readdygpu_b200 as R
    names = declared("readdy_b200.h")
    assert len(names) >= 18
    for n in names:
        assert hasattr(R.lib, n), n


def test_workloads_exports():
    lib = C.CDLL(os.path.join(ROOT, "readdygpu_b200", "libreaddy_workloads.so"))
    for n in declared("readdy_b200_workloads.h"):
        assert hasattr(lib, n), n


def test_desc_layout_matches_header():
    # sizes of the C structs as the compiler lays them out
    from readdygpu_b200 import _abi as A
    assert C.sizeof(A.PairPot) == 4 + 4 + 8 * 4 + 256
    assert C.sizeof(A.Box) == 6 * 8 + 3 * 4 + 4 + 8


def test_no_device_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    import readdygpu_b200 as R
    from readdygpu_b200 import configs
    w = configs.config1(n=10)
    with pytest.raises(R.RdgpuError) as e:
        R.Engine(w.system)
    assert e.value.code == R._abi.ERR_CUDA
    assert "no CPU fallback" in str(e.value)
