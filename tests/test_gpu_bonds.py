"""Bonded pairs of particle groups (rdgpu_set_bonds) against the oracle
(orc_bond_forces_f64): each bond one pair potential at any distance."""
import numpy as np
import pytest

from readdygpu_b200 import _abi as A
from readdygpu_b200.system import System, PairPotential

from .test_gpu_parity import Engine, cfg1, oracle_state

pytestmark = pytest.mark.gpu

POTS = [PairPotential(A.P2_HARMONIC, [], 20.0, "spring"),
        PairPotential(A.P2_HARMONIC, [], 5.0, "attractive", r0=4.2),
        PairPotential(A.P2_WEAK_PIECEWISE, [], 10.0, r0=3.0, length=2.0, depth=1.5)]


def bonds_for(n, nb, seed=3):
    rng = np.random.default_rng(seed)
    ij = set()
    while len(ij) < nb:
        i, j = rng.integers(0, n, 2)
        if i != j:
            ij.add((min(i, j), max(i, j)))
    ij = np.array(sorted(ij), np.int32)
    pot = rng.integers(0, len(POTS), len(ij)).astype(np.int32)
    return ij, pot


def oracle_forces(oracle, sys_, x, types, ij, pot):
    d, stored, _ = oracle_state(oracle, sys_, x, "f64")
    F, E = oracle.forces_f64(d, stored, types)
    pots = [System.pot_struct(p) for p in POTS]
    return oracle.bond_forces(d, stored, types, ij, pot, pots, F, E)


@pytest.mark.parametrize("prec", ["f64", "f32c"])
@pytest.mark.parametrize("mode", ["cells", "list"])
def test_bond_forces_match_oracle(oracle, prec, mode):
    sys_, xyz, types = cfg1(1000)
    ij, pot = bonds_for(1000, 300)
    with Engine(sys_, precision=prec, neighbour_mode=mode, skin=0.7) as e:
        e.set_particles(xyz, types)
        e.set_bonds(ij, pot, POTS)
        e.step(30)
        x1, t1 = e.get_particles()
        F, En = e.forces()
    Fo, Eo = oracle_forces(oracle, sys_, x1, t1, ij, pot)
    rel = np.linalg.norm(F - Fo) / np.linalg.norm(Fo)
    assert rel <= (1e-12 if prec == "f64" else 1e-5), rel
    assert abs(En - Eo) <= (1e-10 if prec == "f64" else 1e-5) * abs(Eo)


def test_bond_step_with_injected_noise(oracle):
    """One FP64 step with bonds: x + a F + b xi with the oracle's forces."""
    sys_, xyz, types = cfg1(800)
    ij, pot = bonds_for(800, 200, seed=5)
    noise = np.random.default_rng(9).standard_normal((800, 3))
    with Engine(sys_, precision="f64", neighbour_mode="cells") as e:
        e.set_particles(xyz, types)
        e.set_bonds(ij, pot, POTS)
        x0, _ = e.get_particles()
        e.step_with_noise(noise)
        x1, _ = e.get_particles()
    Fo, _ = oracle_forces(oracle, sys_, x0, types, ij, pot)
    D = np.array([t.D for t in sys_.types])[types]
    a = (D * sys_.dt / (sys_.kB * sys_.T))[:, None]
    b = np.sqrt(2.0 * D * sys_.dt)[:, None]
    L = np.array(sys_.box_lengths())
    xe = np.mod(x0 + a * Fo + b * noise, L)
    d = x1 - xe
    d -= L * np.round(d / L)
    assert np.abs(d).max() <= 1e-10, np.abs(d).max()


def test_bond_trajectories_cells_list_identical():
    sys_, xyz, types = cfg1(1500)
    ij, pot = bonds_for(1500, 500, seed=7)
    out = []
    for mode in ("cells", "list"):
        with Engine(sys_, precision="f32c", seed=12, neighbour_mode=mode, skin=0.5) as e:
            e.set_particles(xyz, types)
            e.set_bonds(ij, pot, POTS)
            e.step(230)
            out.append(e.get_particles()[0])
    np.testing.assert_array_equal(out[0], out[1])


@pytest.mark.parametrize("mode", ["cells", "list"])
def test_bonds_follow_reaction_edits(oracle, mode):
    sys_, xyz, types = cfg1(600)
    ij, pot = bonds_for(600, 200, seed=11)
    dele = [int(ij[0, 0]), int(ij[5, 1]), 599]
    with Engine(sys_, precision="f64", neighbour_mode=mode, skin=0.6) as e:
        e.set_particles(xyz, types)
        e.set_bonds(ij, pot, POTS)
        e.step(20)
        rows = [[0, -1, 0, 0, 0, g] for g in dele] + [[0, 1, 10.0, 10.0, 10.0, -1]]
        e.apply_edits(np.array(rows, np.float32))
        x2, t2 = e.get_particles()
        F, _ = e.forces()
    keep = np.ones(600, bool)
    keep[dele] = False
    nid = np.cumsum(keep) - 1
    ok = keep[ij[:, 0]] & keep[ij[:, 1]]
    ij2 = np.stack([nid[ij[ok, 0]], nid[ij[ok, 1]]], 1).astype(np.int32)
    Fo, _ = oracle_forces(oracle, sys_, x2, t2, ij2, pot[ok])
    assert np.linalg.norm(F - Fo) <= 1e-10 * np.linalg.norm(Fo)


def test_bond_errors():
    sys_, xyz, types = cfg1(100)
    with Engine(sys_, precision="f64") as e:
        e.set_particles(xyz, types)
        for ij, pot in (([[0, 100]], [0]), ([[3, 3]], [0]), ([[0, 1]], [3])):
            with pytest.raises(RuntimeError):
                e.set_bonds(np.array(ij), np.array(pot), POTS)
