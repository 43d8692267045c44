"""rdgpu_rdf_counts_noalloc: RDF pair counts for callers that cannot allocate
device memory (for example a host runtime that owns the device memory pool
and hands the library its buffers).  The entry point works in a fixed static
device scratch array; these tests check that it gives exactly the counts of
the allocating entry point rdgpu_rdf, call after call, and that it rejects
inputs beyond its stated limits.

This file is collected last on purpose: a failure here leaves every other
test already run.
"""
import ctypes as C

import numpy as np
import pytest

from readdygpu_b200 import _abi as A
from readdygpu_b200.system import System, ParticleType, PairPotential, ExternalPotential


def _system(kind):
    rng = np.random.default_rng(7 if kind == "periodic" else 8)
    if kind == "periodic":
        sys_ = System([ParticleType("A", 1e6, 1.5), ParticleType("B", 5e5, 2.0)],
                      pair=[PairPotential(A.P2_HARMONIC, [(0, 0), (0, 1), (1, 1)], 10.0, "repulsive")],
                      kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(50, 50, 50), periodic=(1, 1, 1))
        xyz = rng.uniform(0, 50, (1500, 3))
        types = rng.integers(0, 2, 1500).astype(np.int32)
    else:
        sys_ = System([ParticleType(f"S{i}", 1e6, 1.0 + 0.5 * i) for i in range(3)],
                      pair=[PairPotential(A.P2_HARMONIC, [(i, j) for i in range(3) for j in range(i, 3)], 10.0,
                                          "repulsive")],
                      external=[ExternalPotential(A.P1_DISK, [2], 10.0, "attractive", radius=20.0)],
                      kT=2.437, dt=1e-9, lo=(-40, -40, -20), hi=(40, 40, 20), periodic=(1, 1, 0))
        xyz = np.column_stack([rng.uniform(-40, 40, 2500), rng.uniform(-40, 40, 2500), rng.uniform(-24, 24, 2500)])
        types = rng.integers(0, 3, 2500).astype(np.int32)
    return sys_, xyz, types


def _noalloc_counts(sys_, xyz, types, nbins, rmax):
    import torch
    import readdygpu_b200 as R
    dev = torch.device("cuda:0")
    x = torch.tensor(np.ascontiguousarray(xyz), dtype=torch.float64, device=dev)
    t = torch.tensor(types, dtype=torch.int32, device=dev)
    S = sys_.n_types
    out = torch.full((S * S * nbins,), -1, dtype=torch.int64, device=dev)   # stale values must be overwritten
    lo = (C.c_double * 3)(*sys_.lo)
    hi = (C.c_double * 3)(*sys_.hi)
    per = (C.c_int32 * 3)(*sys_.periodic)
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = R.lib.rdgpu_rdf_counts_noalloc(x.data_ptr(), t.data_ptr(), len(types), S, lo, hi, per, nbins, rmax,
                                       out.data_ptr(), stream)
    assert rc == 0, R.lib.rdgpu_last_error(None).decode()
    return out.cpu().numpy().view(np.uint64).reshape(S, S, nbins)


def _engine_counts(sys_, xyz, types, nbins, rmax):
    from readdygpu_b200 import Engine
    with Engine(sys_, precision="f64") as e:
        e.set_particles(xyz, types)
        c, _ = e.rdf(nbins, rmax, accumulate=False)
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["periodic", "slab"])
@pytest.mark.parametrize("nbins,rmax", [(60, 12.0), (50, 10.0), (40, 30.0)])
def test_noalloc_matches_rdgpu_rdf_twice(kind, nbins, rmax):
    """rmax 12: cells of 12.5 / 13.3 nm; rmax 10 in the 50 nm box: L / rmax is
    an integer, so the cell edge equals rmax up to rounding, with pairs placed
    just under rmax across cell boundaries; rmax 30: beyond half the box."""
    sys_, xyz, types = _system(kind)
    if rmax == 10.0:
        # pairs just under rmax apart along each axis, straddling cell edges
        ext = []
        for a in range(3):
            for c in (10.0, 20.0, 30.0):
                p = np.array(sys_.lo, dtype=float) + 5.0
                q = p.copy()
                p[a] = sys_.lo[a] + c - 1e-7
                q[a] = p[a] + 10.0 - 1e-6
                ext += [p, q]
        xyz = np.concatenate([xyz, np.array(ext)])
        types = np.concatenate([types, np.zeros(len(ext), np.int32)])
    # two calls in a row, on different particles: the shared scratch keeps the
    # previous call's contents, which must not leak into the next result
    for shift in (0.0, 3.3):
        x = xyz + shift
        got = _noalloc_counts(sys_, x, types, nbins, rmax)
        want = _engine_counts(sys_, x, types, nbins, rmax)
        assert want.sum() > 0
        assert np.array_equal(got, want)


@pytest.mark.gpu
def test_noalloc_rejects_bad_input():
    import readdygpu_b200 as R
    sys_, xyz, types = _system("periodic")
    bad = types.copy()
    bad[5] = 9
    with pytest.raises(AssertionError, match="type out of range"):
        _noalloc_counts(sys_, xyz, bad, 10, 5.0)


def test_noalloc_limits_are_enforced():
    import readdygpu_b200 as R
    lo = (C.c_double * 3)(0, 0, 0)
    hi = (C.c_double * 3)(10, 10, 10)
    per = (C.c_int32 * 3)(1, 1, 1)
    dummy = C.c_void_p(16)      # never dereferenced: the size checks come first
    rc = R.lib.rdgpu_rdf_counts_noalloc(dummy, dummy, A_MAX + 1, 1, lo, hi, per, 10, 2.0, dummy, None)
    assert rc == A.ERR_ARG
    assert "exceeds the maximum" in R.lib.rdgpu_last_error(None).decode()
    rc = R.lib.rdgpu_rdf_counts_noalloc(dummy, dummy, 10, 1, lo, hi, per, 100000, 2.0, dummy, None)
    assert rc == A.ERR_ARG and "nbins" in R.lib.rdgpu_last_error(None).decode()


A_MAX = 65536
