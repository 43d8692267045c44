"""The oracle's bond forces: single-bond closed forms and finite differences."""
import numpy as np

from readdygpu_b200 import _abi as A
from readdygpu_b200.system import System, ParticleType, PairPotential


def two_particle_system():
    return System([ParticleType("A", 1e6, 1.0)], pair=[], kT=2.437, dt=1e-9,
                  lo=(0, 0, 0), hi=(20, 20, 20), periodic=(1, 1, 1))


def test_spring_bond_closed_form(oracle):
    s = two_particle_system()
    d = s.to_desc()
    x = np.array([[1.0, 1.0, 1.0], [18.5, 1.0, 1.0]])      # 2.5 apart through the boundary
    pots = [System.pot_struct(PairPotential(A.P2_HARMONIC, [], 20.0, "spring"))]
    F, E = oracle.bond_forces(d, x, np.zeros(2, np.int32), [[0, 1]], [0], pots)
    # r0 = 1 + 1 = 2, r = 2.5: |F| = k (r - r0) = 10, pulling 0 towards -x (its partner's image)
    np.testing.assert_allclose(F[0], [-10.0, 0, 0], atol=1e-12)
    np.testing.assert_allclose(F[1], [10.0, 0, 0], atol=1e-12)
    assert abs(E - 0.5 * 20.0 * 0.25) < 1e-12


def test_bond_forces_are_energy_gradients(oracle):
    s = two_particle_system()
    d = s.to_desc()
    rng = np.random.default_rng(2)
    x = rng.uniform(5, 15, (6, 3))
    types = np.zeros(6, np.int32)
    pots = [System.pot_struct(p) for p in (
        PairPotential(A.P2_HARMONIC, [], 20.0, "spring"),
        PairPotential(A.P2_WEAK_PIECEWISE, [], 10.0, r0=3.0, length=4.0, depth=1.5))]
    ij = [[0, 1], [1, 2], [3, 4], [4, 5], [0, 5]]
    pot = [0, 1, 0, 1, 1]
    F, _ = oracle.bond_forces(d, x, types, ij, pot, pots)
    h = 1e-6
    for i in range(6):
        for a in range(3):
            xp = x.copy(); xp[i, a] += h
            xm = x.copy(); xm[i, a] -= h
            ep = oracle.bond_forces(d, xp, types, ij, pot, pots)[1]
            em = oracle.bond_forces(d, xm, types, ij, pot, pots)[1]
            assert abs(-(ep - em) / (2 * h) - F[i, a]) < 1e-5
