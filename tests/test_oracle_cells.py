"""CPU checks of the oracle's large-system helpers: the cell-list neighbour
digest (used by the full-size parity tests) equals the brute-force digest bit
for bit, and the oracle's copy of the config-3 input generator (used by the
benchmark's reference arm) gives the engine package's coordinates."""
import numpy as np
import pytest

from readdygpu_b200 import _abi as A
from readdygpu_b200 import configs
from readdygpu_b200.system import System, ParticleType, PairPotential


def _system(lo, hi, per):
    return System([ParticleType("A", 1e6, 1.5), ParticleType("B", 5e5, 2.0), ParticleType("C", 1e6, 0.5)],
                  pair=[PairPotential(A.P2_HARMONIC, [(0, 0), (0, 1), (1, 1)], 10.0, "repulsive"),
                        PairPotential(A.P2_WEAK_PIECEWISE, [(1, 2)], 10.0, r0=2.75, length=1.0, depth=2.0)],
                  kT=2.437, dt=1e-9, lo=lo, hi=hi, periodic=per)


CASES = {
    "periodic": ((0, 0, 0), (40, 40, 40), (1, 1, 1)),
    "z_open": ((-30, -30, -10), (30, 30, 10), (1, 1, 0)),
    "small_periodic": ((0, 0, 0), (9, 30, 30), (1, 1, 1)),     # fewer than 3 cells along x
}


@pytest.mark.parametrize("f32", [False, True])
@pytest.mark.parametrize("case", list(CASES))
def test_cell_digest_equals_brute_force(oracle, case, f32):
    lo, hi, per = CASES[case]
    sys_ = _system(lo, hi, per)
    d = sys_.to_desc()
    rng = np.random.default_rng(3)
    n = 3000
    xyz = rng.uniform(lo, hi, size=(n, 3))
    if not per[2]:
        xyz[:40, 2] = hi[2] + rng.uniform(0, 3, 40)      # beyond the open z bound
    types = rng.integers(0, 3, n).astype(np.int32)
    if f32:
        x, _ = oracle.to_rel_f32(d, xyz)
    else:
        x = oracle.to_rel_f64(d, xyz)
    c0, h0 = oracle.neighbor_digest(d, x, types, f32=f32)
    for threads in (1, 4):
        c1, h1 = oracle.neighbor_digest_cells(d, x, types, f32=f32, threads=threads)
        assert np.array_equal(c0, c1) and np.array_equal(h0, h1)
    assert c0.sum() > 0


def test_oracle_rsa_equals_engine_generator(oracle):
    a = configs.rsa_spheres(2000, 60.0, 4.0, 17)
    b = oracle.rsa_spheres(2000, 60.0, 4.0, 17)
    assert np.array_equal(a, b)
