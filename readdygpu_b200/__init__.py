"""readdygpu_b200 -- B200-native Brownian-dynamics hot path of ReaDDy.

The compute lives in the in-tree shared library libreaddy_b200.so (hand-written
sm_100a CUDA behind the C ABI of include/readdy_b200.h).  There is no CPU
fallback: importing the package fails loudly when the library is missing, and
every compute call fails when no CUDA device is present.
"""
import ctypes as _C
import os as _os

from . import _abi

_HERE = _os.path.dirname(_os.path.abspath(__file__))
LIB_PATH = _os.path.join(_HERE, "libreaddy_b200.so")

if not _os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python readdygpu_b200/build.py` "
        "(there is no CPU fallback)")

lib = _abi.bind(_C.CDLL(LIB_PATH))

from .system import (System, ParticleType, PairPotential, ExternalPotential,  # noqa: E402
                     float_exact_box)
from .engine import Engine, RdgpuError  # noqa: E402

__all__ = ["lib", "LIB_PATH", "System", "ParticleType", "PairPotential", "ExternalPotential",
           "Engine", "RdgpuError", "float_exact_box"]
