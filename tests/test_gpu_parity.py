"""GPU parity: the sm_100a engine (through the C ABI) against the CPU oracle.

Bars (stated per test):
  * neighbour sets and RDF counts: bit-exact (same predicate arithmetic);
  * FP64 forces: relative 1e-12 (norm-wise), positions after a step 1e-11 nm;
  * FP32-compensated forces: ||F32 - F64|| / ||F64|| <= 1e-5 and per particle
    |dF| <= 1e-5 |F| + 2e-5 kJ/mol/nm; positions after a step 2e-6 nm;
  * the reference's own displacement KATs: 1e-4 (their JUnit tolerance).
"""
import json
import math
import os

import numpy as np
import pytest

from readdygpu_b200 import _abi as A
from readdygpu_b200.system import System, ParticleType, PairPotential, ExternalPotential, float_exact_box

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
PRECS = ["f64", "f32c"]


def Engine(*a, **k):
    from readdygpu_b200 import Engine as E
    return E(*a, **k)


def small_config2(n=4000, seed=11):
    """config 2's potentials (4 species, weak interaction, disk, z non-periodic)
    in a smaller box."""
    rng = np.random.default_rng(seed)
    radii = [1.0, 1.5, 2.0, 3.0]
    D = [1e5, 1e6, 3e6, 1e7]
    s01 = 2.5
    sys_ = System([ParticleType(f"S{i}", D[i], radii[i]) for i in range(4)],
                  pair=[PairPotential(A.P2_HARMONIC, [(i, j) for i in range(4) for j in range(i, 4)], 10.0, "repulsive"),
                        PairPotential(A.P2_WEAK_PIECEWISE, [(0, 1)], 10.0, r0=1.1 * s01, length=0.4 * s01, depth=2.0)],
                  external=[ExternalPotential(A.P1_DISK, [3], 10.0, "attractive", center=(0, 0, 0),
                                              normal=(0, 0, 1), radius=20.0)],
                  kT=2.437, dt=1e-9, lo=(-40, -40, -20), hi=(40, 40, 20), periodic=(1, 1, 0))
    xyz = np.column_stack([rng.uniform(-40, 40, n), rng.uniform(-40, 40, n), rng.uniform(-24, 24, n)])
    types = rng.integers(0, 4, n).astype(np.int32)
    return sys_, xyz, types


def cfg1(n=1000):
    from readdygpu_b200 import configs
    w = configs.config1(n=n)
    return w.system, w.xyz, w.types


CASES = {"config1": cfg1, "config2_small": small_config2}


def oracle_state(O, sys_, xyz, prec):
    d = sys_.to_desc()
    if prec == "f64":
        x = O.to_rel_f64(d, xyz).reshape(-1, 3)
        return d, x, x
    hi, comp = O.to_rel_f32(d, xyz)
    return d, hi.reshape(-1, 3), hi.astype(np.float64).reshape(-1, 3) - comp.astype(np.float64).reshape(-1, 3)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("case", list(CASES))
def test_neighbor_sets_bit_exact(oracle, prec, case):
    sys_, xyz, types = CASES[case]()
    d, stored, _ = oracle_state(oracle, sys_, xyz, prec)
    with Engine(sys_, precision=prec) as e:
        e.set_particles(xyz, types)
        cnt, h = e.neighbor_digest()
    ocnt, oh = oracle.neighbor_digest(d, stored, types, f32=(prec == "f32c"))
    assert cnt.sum() > 0
    assert np.array_equal(cnt, ocnt)
    assert np.array_equal(h, oh)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("case", list(CASES))
def test_forces_and_energy(oracle, prec, case):
    sys_, xyz, types = CASES[case]()
    d, stored, _ = oracle_state(oracle, sys_, xyz, prec)
    with Engine(sys_, precision=prec) as e:
        e.set_particles(xyz, types)
        F, E = e.forces()
    Fo, Eo = oracle.forces_f64(d, stored.astype(np.float64), types)
    nrm = np.linalg.norm(Fo)
    assert nrm > 0
    rel = np.linalg.norm(F - Fo) / nrm
    if prec == "f64":
        assert rel <= 1e-12, rel
        assert abs(E - Eo) <= 1e-10 * max(1.0, abs(Eo))
    else:
        assert rel <= 1e-5, rel
        per = np.linalg.norm(F - Fo, axis=1)
        assert np.all(per <= 1e-5 * np.linalg.norm(Fo, axis=1) + 2e-5), per.max()
        assert abs(E - Eo) <= 1e-5 * max(1.0, abs(Eo))


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("case", list(CASES))
def test_step_with_injected_noise(oracle, prec, case):
    sys_, xyz, types = CASES[case]()
    d, _, truth = oracle_state(oracle, sys_, xyz, prec)
    noise = np.random.default_rng(5).standard_normal((types.size, 3))
    with Engine(sys_, precision=prec) as e:
        e.set_particles(xyz, types)
        e.step_with_noise(noise)
        x1, t1 = e.get_particles()
    xo, rc = oracle.step_f64(d, truth, types, noise)
    assert rc == 0
    xo = xo + np.array(sys_.lo)
    L = np.array(sys_.box_lengths())
    dx = x1 - xo
    per = np.array(sys_.periodic, bool)
    dx[:, per] -= L[per] * np.round(dx[:, per] / L[per])
    tol = 1e-11 if prec == "f64" else 2e-6
    assert np.abs(dx).max() <= tol, np.abs(dx).max()
    assert np.array_equal(t1, types)


@pytest.mark.parametrize("prec", PRECS)
def test_philox_noise_matches_oracle(oracle, prec):
    sys_, xyz, types = cfg1(300)
    seed = 987654321
    with Engine(sys_, precision=prec, seed=seed) as e:
        e.set_particles(xyz, types)
        z = e.debug_noise(17)
    zo = np.array([oracle.bd_normals(seed, 17, i) for i in range(types.size)])
    tol = 1e-12 if prec == "f64" else 2e-5
    assert np.abs(z - zo).max() <= tol


def test_fp32_normals_over_many_words(oracle):
    """The FP32 Box-Muller transform over 1.2 M Philox words (200,000
    particles, 2 steps): every normal within 2e-5 of the oracle's FP64 one,
    the words near u = 1 (where the radius is sqrt(-2 ln u) of a small
    logarithm) and near u = 0 included."""
    n = 200_000
    sys_ = System([ParticleType("A", 1e6, 1.0)], pair=[PairPotential(A.P2_HARMONIC, [(0, 0)], 10.0, "repulsive")],
                  kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(300.0, 300.0, 300.0), periodic=(1, 1, 1))
    xyz = np.random.default_rng(8).uniform(0, 300.0, (n, 3))
    seed = 1357911
    with Engine(sys_, precision="f32c", seed=seed, neighbour_mode="cells") as e:
        e.set_particles(xyz, np.zeros(n, np.int32))
        zs = [e.debug_noise(t) for t in (3, 4)]
    for t, z in zip((3, 4), zs):
        zo = oracle.bd_normals_many(seed, t, n)
        err = np.abs(z - zo)
        assert err.max() <= 2e-5, (t, err.max(), zo.ravel()[err.argmax()])
        r2 = zo[:, 0] ** 2 + zo[:, 1] ** 2
        assert r2.min() < 1e-4 and r2.max() > 20.0      # both ends of the radius were drawn


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("nbins,rmax", [(50, 12.0), (64, 30.0)])
def test_rdf_counts_bit_exact(oracle, prec, nbins, rmax):
    sys_, xyz, types = small_config2(3000) if rmax < 20 else cfg1(1000)
    d, stored, _ = oracle_state(oracle, sys_, xyz, prec)
    with Engine(sys_, precision=prec) as e:
        e.set_particles(xyz, types)
        c, frames = e.rdf(nbins, rmax, accumulate=True)
        c2, frames2 = e.rdf(nbins, rmax, accumulate=True)
    co = oracle.rdf_counts(d, stored, types, nbins, rmax, f32=(prec == "f32c"))
    assert frames == 1 and frames2 == 2
    assert c.sum() > 0
    assert np.array_equal(c.ravel(), co)
    assert np.array_equal(c2.ravel(), 2 * co)
    # both orientations of every unordered pair (CudaSimulation.cu:1817-1818)
    assert np.array_equal(c, c.transpose(1, 0, 2))


def ext_system(prec):
    kinds = [(A.P1_DISK, "attractive"), (A.P1_DISK, "repulsive"), (A.P1_CYLINDER, "attractive"),
             (A.P1_CYLINDER, "repulsive"), (A.P1_SPHERE, "attractive"), (A.P1_SPHERE, "repulsive"),
             (A.P1_SPHERE, "membrane"), (A.P1_CUBE, "attractive"), (A.P1_CUBE, "repulsive")]
    types = [ParticleType(f"T{i}", 1e6, 0.5 + 0.25 * i) for i in range(len(kinds))]
    ext = []
    for t, (k, sub) in enumerate(kinds):
        ext.append(ExternalPotential(k, [t], 3.0 + t, sub, center=(1.0, -2.0, 0.5), normal=(1.0, 2.0, 2.0),
                                     radius=6.0, height=5.0, origin=(-8, -7, -6), extension=(15, 14, 13)))
    sys_ = System(types, external=ext, kT=2.437, dt=1e-9, lo=(-16, -16, -16), hi=(16, 16, 16), periodic=(1, 1, 1))
    rng = np.random.default_rng(3)
    n = 450
    xyz = rng.uniform(-15, 15, size=(n, 3))
    tt = (np.arange(n) % len(kinds)).astype(np.int32)
    return sys_, xyz, tt


@pytest.mark.parametrize("prec", PRECS)
def test_external_potentials(oracle, prec):
    sys_, xyz, types = ext_system(prec)
    d, stored, _ = oracle_state(oracle, sys_, xyz, prec)
    with Engine(sys_, precision=prec) as e:
        e.set_particles(xyz, types)
        F, E = e.forces()
    Fo, Eo = oracle.forces_f64(d, stored.astype(np.float64), types)
    nz = np.linalg.norm(Fo, axis=1) > 0
    assert nz.sum() > 100
    tol = 1e-11 if prec == "f64" else 1e-5
    assert np.linalg.norm(F - Fo) <= tol * np.linalg.norm(Fo)
    assert abs(E - Eo) <= tol * 10 * abs(Eo)


# ---- the reference's own displacement KATs, run through the GPU step -----

KATS = json.load(open(os.path.join(HERE, "golden", "reference_kats.json")))


@pytest.mark.parametrize("prec", PRECS)
def test_single_displacement_kats_on_gpu(prec):
    f = KATS["displacement_fixture"]
    for case in KATS["single_displacement"]:
        dk = f["disk"]
        t = ParticleType("A", f["D"][case["type"]], case["p_radius"])
        sys_ = System([t], external=[ExternalPotential(A.P1_DISK, [0], dk["k"], "attractive", center=dk["center"],
                                                       normal=dk["normal"], radius=dk["radius"])],
                      kB=f["Kb"], T=f["T"], dt=f["dt"], lo=(-64, -64, -64), hi=(64, 64, 64), periodic=(1, 1, 1))
        x0 = np.array([case["x"]])
        with Engine(sys_, precision=prec) as e:
            e.set_particles(x0, [0])
            e.step_with_noise(np.zeros(3))
            x1, _ = e.get_particles()
        np.testing.assert_allclose(x1[0] - x0[0], case["disp"], atol=KATS["tolerance"], err_msg=case["where"])


@pytest.mark.parametrize("prec", PRECS)
def test_pair_displacement_kats_on_gpu(prec):
    f = KATS["displacement_fixture"]
    for case in KATS["pair_displacement"]:
        p1, p2 = case["p1"], case["p2"]
        t1, t2 = p1["type"], p2["type"]
        half = case["radius"] / 2.0
        types = [ParticleType("a", f["D"][t1], half), ParticleType("b", f["D"][t2], half)]
        pots = []
        if sorted([t1, t2]) in [sorted(x) for x in f["harmonic_attractive"]["type_pairs"]]:
            pots.append(PairPotential(A.P2_HARMONIC, [(0, 1)], f["harmonic_attractive"]["k"], "attractive"))
        if [p1["id"], p2["id"]] in f["harmonic_repulsive_id"]["id_pairs"]:
            pots.append(PairPotential(A.P2_HARMONIC, [(0, 1)], f["harmonic_repulsive_id"]["k"], "repulsive"))
        if sorted([t1, t2]) in [sorted(x) for x in f["harmonic_spring"]["type_pairs"]]:
            pots.append(PairPotential(A.P2_HARMONIC, [(0, 1)], f["harmonic_spring"]["k"], "spring"))
        sys_ = System(types, pair=pots, kB=f["Kb"], T=f["T"], dt=f["dt"], lo=(-40, -40, -40), hi=(40, 40, 40),
                      periodic=(1, 1, 1), max_cutoff=10.0)
        x0 = np.array([p1["x"], p2["x"]], float)
        with Engine(sys_, precision=prec) as e:
            e.set_particles(x0, [0, 1])
            e.step_with_noise(np.zeros(6))
            x1, _ = e.get_particles()
        np.testing.assert_allclose(x1[0] - x0[0], case["disp1"], atol=KATS["tolerance"], err_msg=case["where"])
        np.testing.assert_allclose(x1[1] - x0[1], case["disp2"], atol=KATS["tolerance"], err_msg=case["where"])


# ---- dynamics: determinism, batching, overflow recovery, MSD --------------

def test_f32_run_is_deterministic():
    sys_, xyz, types = small_config2(3000)
    out = []
    for _ in range(2):
        with Engine(sys_, precision="f32c", seed=42) as e:
            e.set_particles(xyz, types)
            e.step(250)
            out.append(e.get_particles()[0])
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("prec", PRECS)
def test_batch_matches_single_systems(prec):
    from readdygpu_b200 import configs
    w = configs.config4(n_systems=5, steps=30, nmin=300, nmax=3000)
    with Engine(w.system, precision=prec, boxes=w.boxes) as e:
        e.set_particles(w.xyz, w.types, offsets=w.offsets)
        e.step(30)
        xb, _ = e.get_particles()
    for k, (lo, hi, per, sd) in enumerate(w.boxes):
        a, b = w.offsets[k], w.offsets[k + 1]
        s = w.system
        single = System(s.types, pair=s.pair, external=s.external, kB=s.kB, T=s.T, dt=s.dt, lo=lo, hi=hi, periodic=per)
        with Engine(single, precision=prec, seed=sd) as e:
            e.set_particles(w.xyz[a:b], w.types[a:b])
            e.step(30)
            xs, _ = e.get_particles()
        if prec == "f32c":
            assert np.array_equal(xb[a:b], xs)        # fixed-point sums: order independent
        else:
            assert np.abs(xb[a:b] - xs).max() < 1e-9


@pytest.mark.parametrize("prec", PRECS)
def test_dense_cluster(oracle, prec):
    """Hundreds of particles in a few cells (the sorted cell layout has no
    per-cell capacity): neighbour sets stay bit-exact and forces match."""
    rng = np.random.default_rng(21)
    sys_ = System([ParticleType("A", 1e6, 1.0)], pair=[PairPotential(A.P2_HARMONIC, [(0, 0)], 10.0, "repulsive")],
                  kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(40, 40, 40), periodic=(1, 1, 1))
    xyz = np.concatenate([rng.uniform(0, 40, (300, 3)), 20.0 + rng.uniform(-1.5, 1.5, (400, 3))])
    types = np.zeros(len(xyz), np.int32)
    d, stored, _ = oracle_state(oracle, sys_, xyz, prec)
    with Engine(sys_, precision=prec) as e:
        e.set_particles(xyz, types)
        cnt, h = e.neighbor_digest()
        F, _ = e.forces()
        e.step(20)
    ocnt, oh = oracle.neighbor_digest(d, stored, types, f32=(prec == "f32c"))
    assert cnt.max() > 300
    assert np.array_equal(cnt, ocnt) and np.array_equal(h, oh)
    Fo, _ = oracle.forces_f64(d, stored.astype(np.float64), types)
    assert np.linalg.norm(F - Fo) <= (1e-12 if prec == "f64" else 1e-5) * np.linalg.norm(Fo)


@pytest.mark.parametrize("prec", PRECS)
def test_msd_matches_positions(prec):
    sys_, xyz, types = cfg1(1000)
    with Engine(sys_, precision=prec, seed=3) as e:
        e.set_particles(xyz, types)
        x0, _ = e.get_particles()
        e.step(200)
        x1, _ = e.get_particles()
        m = e.metrics()
    d = x1 - x0
    d -= 50.0 * np.round(d / 50.0)
    for t in (0, 1):
        want = (d[types == t] ** 2).sum(1).mean()
        assert abs(m["msd"][t] - want) <= 1e-6 * want
        assert m["count"][t] == (types == t).sum()
    # diffusion: MSD ~ 6 D t (within noise and the repulsion's slowdown)
    t_tot = 200 * 1e-9
    assert 0.5 < m["msd"][0] / (6 * 1e6 * t_tot) < 1.3


@pytest.mark.parametrize("prec", PRECS)
def test_energy_metric_matches_forces_energy(prec):
    sys_, xyz, types = small_config2(2000)
    with Engine(sys_, precision=prec) as e:
        e.set_particles(xyz, types)
        _, E = e.forces()
        m = e.metrics()
    assert m["energy"] == E


# ---- edge cases -----------------------------------------------------------

@pytest.mark.parametrize("prec", PRECS)
def test_small_periodic_boxes_dedupe_cells(oracle, prec):
    """fewer than 3 cells along an axis: each neighbour cell is visited once
    (the reference double counts there, CudaSimulation.cu:1333-1396)."""
    rng = np.random.default_rng(9)
    for L in (8.0, 12.0):           # 2 and 3 cells of >= 4 nm
        sys_ = System([ParticleType("A", 1e6, 2.0)], pair=[PairPotential(A.P2_HARMONIC, [(0, 0)], 10.0, "repulsive")],
                      kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(L, L, 40.0), periodic=(1, 1, 1))
        xyz = rng.uniform(0, 1, (60, 3)) * np.array([L, L, 40.0])
        types = np.zeros(60, np.int32)
        d, stored, _ = oracle_state(oracle, sys_, xyz, prec)
        with Engine(sys_, precision=prec) as e:
            e.set_particles(xyz, types)
            cnt, h = e.neighbor_digest()
            F, _ = e.forces()
        ocnt, oh = oracle.neighbor_digest(d, stored, types, f32=(prec == "f32c"))
        assert np.array_equal(cnt, ocnt) and np.array_equal(h, oh)
        Fo, _ = oracle.forces_f64(d, stored.astype(np.float64), types)
        assert np.linalg.norm(F - Fo) <= (1e-12 if prec == "f64" else 1e-5) * np.linalg.norm(Fo)


@pytest.mark.parametrize("prec", PRECS)
def test_empty_and_single_particle(prec):
    sys_, _, _ = cfg1(10)
    with Engine(sys_, precision=prec) as e:
        e.set_particles(np.zeros((0, 3)), np.zeros(0, np.int32))
        e.step(5)
        e.set_particles(np.array([[25.0, 25.0, 25.0]]), [1])
        e.step(10)
        x, t = e.get_particles()
        assert x.shape == (1, 3) and t[0] == 1
        F, E = e.forces()
        assert np.all(F == 0) and E == 0


@pytest.mark.parametrize("prec", PRECS)
def test_errors_are_reported(prec):
    from readdygpu_b200 import RdgpuError
    sys_, xyz, types = cfg1(50)
    with Engine(sys_, precision=prec) as e:
        with pytest.raises(RdgpuError) as ex:
            e.set_particles(xyz, np.full(50, 7, np.int32))
        assert ex.value.code == A.ERR_ARG
        bad = xyz.copy()
        bad[3, 1] = np.nan
        with pytest.raises(RdgpuError):
            e.set_particles(bad, types)
        with pytest.raises(RdgpuError) as ex:
            e.step(1)
        assert ex.value.code == A.ERR_STATE
    tiny = System(sys_.types, pair=sys_.pair, kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(6, 50, 50), periodic=(1, 1, 1))
    with pytest.raises(RdgpuError):
        Engine(tiny, precision=prec)
