"""readdygpu_b200 -- B200-native Brownian-dynamics hot path of ReaDDy.

The compute lives in the in-tree shared library libreaddy_b200.so (hand-written
sm_100a CUDA behind the C ABI of include/readdy_b200.h).  It is mapped on first
use (`readdygpu_b200.lib`, or the first Engine), so that the host-side
descriptions (System, the benchmark workloads) import without it.  There is no
CPU fallback: that first use raises ImportError when the library is missing,
and every compute call fails when no CUDA device is present.
"""
import ctypes as _C
import os as _os

from . import _abi
from .system import (System, ParticleType, PairPotential, ExternalPotential,  # noqa: E402
                     float_exact_box)
from .engine import Engine, RdgpuError  # noqa: E402

_HERE = _os.path.dirname(_os.path.abspath(__file__))
LIB_PATH = _os.path.join(_HERE, "libreaddy_b200.so")
_LIB = None


def load():
    """The engine library (ctypes, signatures bound), mapped on the first call."""
    global _LIB
    if _LIB is None:
        if not _os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python readdygpu_b200/build.py` "
                "(there is no CPU fallback)")
        _LIB = _abi.bind(_C.CDLL(LIB_PATH))
    return _LIB


def __getattr__(name):
    if name == "lib":
        return load()
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")


__all__ = ["lib", "load", "LIB_PATH", "System", "ParticleType", "PairPotential", "ExternalPotential",
           "Engine", "RdgpuError", "float_exact_box"]
