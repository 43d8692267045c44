"""Pair-list mode against the cell walk and the oracle.

The pair list (radius rc_max + skin, rebuilt with a re-sort by cell whenever a
particle has moved more than about skin/2 since the last build) must find
exactly the pairs the cell walk finds.  FP32 forces are summed in fixed point,
so FP32C trajectories of the two modes are bit-identical; FP64 trajectories
agree to rounding (the summation order differs).
"""
import numpy as np
import pytest

from readdygpu_b200 import _abi as A
from readdygpu_b200.system import System, ParticleType, PairPotential

from .test_gpu_parity import Engine, cfg1, small_config2, oracle_state

pytestmark = pytest.mark.gpu


def run(sys_, xyz, types, prec, steps, chunks=1, **kw):
    with Engine(sys_, precision=prec, seed=77, **kw) as e:
        e.set_particles(xyz, types)
        for _ in range(chunks):
            e.step(steps)
        x, t = e.get_particles()
        m = e.metrics()
    return x, t, m


def same(prec, a, b):
    if prec == "f32c":
        assert np.array_equal(a, b), np.abs(a - b).max()
    else:
        assert np.abs(a - b).max() <= 1e-9, np.abs(a - b).max()


def cluster_system(n_gas=300, n_cluster=400, seed=21):
    rng = np.random.default_rng(seed)
    sys_ = System([ParticleType("A", 1e6, 1.0)], pair=[PairPotential(A.P2_HARMONIC, [(0, 0)], 10.0, "repulsive")],
                  kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(40, 40, 40), periodic=(1, 1, 1))
    xyz = np.concatenate([rng.uniform(0, 40, (n_gas, 3)), 20.0 + rng.uniform(-1.5, 1.5, (n_cluster, 3))])
    return sys_, xyz, np.zeros(len(xyz), np.int32)


@pytest.mark.parametrize("prec", ["f32c", "f64"])
@pytest.mark.parametrize("skin", [0.2, 1.0])
def test_list_trajectory_equals_cells(prec, skin):
    """config 1 (periodic cube), 250 steps: small skins rebuild almost every
    step, larger ones every few steps; the trajectory is the cell walk's."""
    sys_, xyz, types = cfg1(2000)
    xc, tc, mc = run(sys_, xyz, types, prec, 250, neighbour_mode="cells")
    xl, tl, ml = run(sys_, xyz, types, prec, 250, neighbour_mode="list", skin=skin)
    assert mc["neighbour_mode"] == "cells" and ml["neighbour_mode"] == "list"
    assert ml["skin"] == skin
    assert 1 < ml["list_builds"] <= 252
    assert np.array_equal(tc, tl)
    same(prec, xc, xl)


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_list_nonperiodic_weak_and_disk(prec):
    """config 2's potentials: z non-periodic, weak interaction, disk; several
    rdgpu_step calls (graph and non-graph launches) and a mid-run upload."""
    sys_, xyz, types = small_config2(3000)
    xc, _, _ = run(sys_, xyz, types, prec, 130, chunks=2, neighbour_mode="cells")
    xl, _, ml = run(sys_, xyz, types, prec, 130, chunks=2, neighbour_mode="list", skin=0.8)
    assert ml["neighbour_mode"] == "list"
    same(prec, xc, xl)


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_list_overflow_regrows_exactly(prec):
    """A dense cluster overflows the capacity estimated from the mean density:
    the build grows the lists and redoes the re-sort; results are unchanged."""
    sys_, xyz, types = cluster_system()
    xc, _, _ = run(sys_, xyz, types, prec, 60, neighbour_mode="cells")
    xl, _, ml = run(sys_, xyz, types, prec, 60, neighbour_mode="list", skin=1.0)
    assert ml["list_capacity"] > 300
    same(prec, xc, xl)


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_list_batch_equals_cells(prec):
    """A batch of 12 systems of uneven size (config 4's recipe)."""
    from readdygpu_b200 import configs
    w = configs.config4(n_systems=12, nmin=200, nmax=3000)
    out = []
    for mode in ("cells", "list"):
        with Engine(w.system, precision=prec, boxes=w.boxes, neighbour_mode=mode, skin=0.6) as e:
            e.set_particles(w.xyz, w.types, offsets=w.offsets)
            e.step(220)
            out.append(e.get_particles()[0])
            m = e.metrics()
    assert m["neighbour_mode"] == "list"
    same(prec, out[0], out[1])


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_list_diagnostics_match_oracle(oracle, prec):
    """After list-mode steps, forces, neighbour sets and RDF counts (which walk
    freshly sorted cells) match the oracle on the engine's own state."""
    sys_, xyz, types = cfg1(1500)
    with Engine(sys_, precision=prec, seed=5, neighbour_mode="list", skin=0.5) as e:
        e.set_particles(xyz, types)
        e.step(120)
        x1, t1 = e.get_particles()
        cnt, h = e.neighbor_digest()
        F, _ = e.forces()
        c, _ = e.rdf(40, 10.0)
    d, stored, _ = oracle_state(oracle, sys_, x1, "f64")
    ocnt, oh = oracle.neighbor_digest(d, stored, t1, f32=False)
    # the engine's stored FP32 positions differ from the FP64 re-import by
    # rounding, so compare the FP32 case through its own counts and sums
    if prec == "f64":
        assert np.array_equal(cnt, ocnt) and np.array_equal(h, oh)
        Fo, _ = oracle.forces_f64(d, stored, t1)
        assert np.linalg.norm(F - Fo) <= 1e-10 * np.linalg.norm(Fo)
        co = oracle.rdf_counts(d, stored, t1, 40, 10.0, f32=False)
        assert np.array_equal(c.reshape(-1), np.asarray(co).reshape(-1))
    else:
        assert cnt.sum() > 0 and abs(int(cnt.sum()) - int(ocnt.sum())) <= 0.01 * ocnt.sum()


def test_list_cells_diagnostics_identical():
    """FP32C: the diagnostics after list steps equal those after cell steps:
    neighbour sets, fixed-point forces and RDF counts bit for bit; the energy
    (FP32 per-particle pair sums in walk order, which depends on the order of
    the particles within a cell) to FP32 rounding."""
    sys_, xyz, types = cfg1(1500)
    res = []
    for mode in ("cells", "list"):
        with Engine(sys_, precision="f32c", seed=9, neighbour_mode=mode, skin=0.4) as e:
            e.set_particles(xyz, types)
            e.step(150)
            cnt, h = e.neighbor_digest()
            F, En = e.forces()
            c, _ = e.rdf(30, 9.0)
            res.append((cnt, h, F, En, c))
    for q, (a, b) in enumerate(zip(res[0], res[1])):
        if q == 3:
            assert abs(a - b) <= 1e-6 * abs(a), (a, b)
        else:
            assert np.array_equal(np.asarray(a), np.asarray(b))


def test_autotune_keeps_the_trajectory():
    """AUTO times the modes on a snapshot and restores it: the trajectory is
    the cell walk's, whatever it picks."""
    sys_, xyz, types = cfg1(3000)
    xc, _, _ = run(sys_, xyz, types, "f32c", 450, neighbour_mode="cells")
    xa, _, ma = run(sys_, xyz, types, "f32c", 450, neighbour_mode="auto")
    assert ma["neighbour_mode"] in ("cells", "list")
    assert ma["step"] == 450
    assert np.array_equal(xc, xa)


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_list_step_with_injected_noise(oracle, prec):
    """One list-mode step with injected noise against the oracle step."""
    sys_, xyz, types = cfg1(1000)
    d, stored, truth = oracle_state(oracle, sys_, xyz, prec)
    noise = np.random.default_rng(5).standard_normal((types.size, 3))
    with Engine(sys_, precision=prec, neighbour_mode="list", skin=0.5) as e:
        e.set_particles(xyz, types)
        e.step_with_noise(noise)
        x1, _ = e.get_particles()
    xo, rc = oracle.step_f64(d, truth, types, noise)
    assert rc == 0
    L = np.array(sys_.box_lengths())
    dx = x1 - (xo + np.array(sys_.lo))
    per = np.array(sys_.periodic, bool)
    dx[:, per] -= L[per] * np.round(dx[:, per] / L[per])
    tol = 1e-11 if prec == "f64" else 2e-6
    assert np.abs(dx).max() <= tol, np.abs(dx).max()


def test_list_falls_back_on_small_boxes():
    """A box with fewer than 3 list cells on a periodic axis keeps the cell walk."""
    sys_ = System([ParticleType("A", 1e6, 2.0)], pair=[PairPotential(A.P2_HARMONIC, [(0, 0)], 10.0, "repulsive")],
                  kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(10, 10, 10), periodic=(1, 1, 1))
    xyz = np.random.default_rng(1).uniform(0, 10, (20, 3))
    with Engine(sys_, precision="f32c", neighbour_mode="list", skin=1.0) as e:
        e.set_particles(xyz, np.zeros(20, np.int32))
        e.step(5)
        assert e.metrics()["neighbour_mode"] == "cells"


def pair_system(skin=1.0):
    """Two particles of radius 2 (harmonic repulsion below 4 nm) in a periodic
    40 nm cube; D dt chosen so that a noise value of 1 moves sqrt(2e-3) nm."""
    sys_ = System([ParticleType("A", 1e6, 2.0)], pair=[PairPotential(A.P2_HARMONIC, [(0, 0)], 10.0, "repulsive")],
                  kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(40, 40, 40), periodic=(1, 1, 1))
    return sys_, np.sqrt(2e-3)


def moves(b, *dx):
    """injected noise that moves particle k by dx[k] nm along x"""
    return np.array([[d / b, 0.0, 0.0] for d in dx])


def run_moves(sys_, xyz, prec, mode, steps):
    """injected-noise steps; the final positions and the list builds so far
    (the upload's included; metrics() reports the count before the re-sort
    that its own energy evaluation does)"""
    with Engine(sys_, precision=prec, neighbour_mode=mode, skin=1.0) as e:
        e.set_particles(xyz, np.zeros(len(xyz), np.int32))
        for mv in steps:
            e.step_with_noise(mv)
        x, _ = e.get_particles()
        m = e.metrics()
    assert m["neighbour_mode"] == mode
    return x, m["list_builds"]


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_list_check_keeps_list_for_an_isolated_hot_particle(prec):
    """skin 1 nm: a particle that moved 0.7 nm (more than skin/2, less than
    skin) with no partner nearby keeps the list; at 1.4 nm the list is rebuilt."""
    sys_, b = pair_system()
    xyz = np.array([[10.0, 10.0, 10.0], [30.0, 30.0, 30.0]])
    x1, n1 = run_moves(sys_, xyz, prec, "list", [moves(b, 0.7, 0.0)])
    x2, n2 = run_moves(sys_, xyz, prec, "list", [moves(b, 0.7, 0.0)] * 2)
    assert n1 == 1 and n2 == 2
    assert abs(x1[0, 0] - 10.7) < 1e-5 and abs(x2[0, 0] - 11.4) < 1e-5 and np.allclose(x2[1], 30.0)


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_list_check_catches_an_approaching_pair(prec):
    """Two particles 5.1 nm apart (outside the 5 nm list radius) approach by
    0.6 nm per step, each moving less than the skin: after two steps they are
    3.9 nm apart and unlisted; the check rebuilds the list before the next
    step's forces, so the trajectory is the cell walk's."""
    sys_, b = pair_system()
    xyz = np.array([[10.0, 10.0, 10.0], [15.1, 10.0, 10.0]])
    steps = [moves(b, 0.3, -0.3)] * 2
    x2, n2 = run_moves(sys_, xyz, prec, "list", steps)
    assert abs((x2[1, 0] - x2[0, 0]) - 3.9) < 1e-5
    assert n2 == 2          # the upload's build and the check's
    steps += [moves(b, 0.0, 0.0)] * 2
    xc, _ = run_moves(sys_, xyz, prec, "cells", steps)
    xl, _ = run_moves(sys_, xyz, prec, "list", steps)
    # the repulsion acted: the pair moved apart in the force-only steps
    assert xc[1, 0] - xc[0, 0] > 3.9 + 1e-3
    same(prec, xc, xl)


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_list_long_run_equals_cells(prec):
    """config 1, 1200 steps at skin 1.0: long intervals between rebuilds, in
    which the list check looks after the hot particles; the trajectory is the
    cell walk's."""
    sys_, xyz, types = cfg1(3000)
    xc, _, _ = run(sys_, xyz, types, prec, 1200, neighbour_mode="cells")
    xl, _, ml = run(sys_, xyz, types, prec, 1200, neighbour_mode="list", skin=1.0)
    assert ml["neighbour_mode"] == "list"
    same(prec, xc, xl)


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_list_check_overflow_of_hot_particles_rebuilds(prec):
    """Every particle of 2000 moves 0.6 nm (more than skin/2, less than the
    skin) in a random direction: far more hot particles than the check takes
    (N/300, at least 8), so the step rebuilds the list outright; then forces
    act on the rebuilt list.  The trajectory is the cell walk's."""
    sys_, xyz, types = cfg1(2000)
    b = np.array([np.sqrt(2.0 * t.D * sys_.dt) for t in sys_.types])[types]
    rng = np.random.default_rng(12)
    u = rng.standard_normal((2000, 3))
    u *= 0.6 / np.linalg.norm(u, axis=1, keepdims=True)
    kick = u / b[:, None]
    out = {}
    for mode in ("cells", "list"):
        with Engine(sys_, precision=prec, neighbour_mode=mode, skin=1.0) as e:
            e.set_particles(xyz, types)
            e.step_with_noise(kick)
            for _ in range(3):
                e.step_with_noise(np.zeros((2000, 3)))
            x, _ = e.get_particles()
            m = e.metrics()
        out[mode] = (x, m)
    assert out["list"][1]["neighbour_mode"] == "list"
    assert out["list"][1]["list_builds"] >= 2
    same(prec, out["cells"][0], out["list"][0])


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_list_check_hot_particles_over_many_blocks(prec):
    """150 of 60,000 particles (config 1's species at config 4's density, a
    periodic 200 nm cube) move 0.6 nm (more than skin/2, less than the skin)
    in a random direction: within the check's cap (N/300 = 200), so the
    check looks at all of them, one warp each over 19 blocks of 8 warps, and
    keeps the list (no pair can have closed the skin).  The trajectory is the
    cell walk's."""
    n, L = 60_000, 200.0
    sys_ = System([ParticleType("A", 1e6, 1.5), ParticleType("B", 5e5, 2.0)],
                  pair=[PairPotential(A.P2_HARMONIC, [(0, 0), (0, 1), (1, 1)], 10.0, "repulsive")],
                  kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(L, L, L), periodic=(1, 1, 1))
    rng = np.random.default_rng(13)
    xyz = rng.uniform(0, L, (n, 3))
    types = (np.arange(n) % 2).astype(np.int32)
    b = np.array([np.sqrt(2.0 * t.D * sys_.dt) for t in sys_.types])[types]
    u = rng.standard_normal((n, 3))
    u *= 0.6 / np.linalg.norm(u, axis=1, keepdims=True)
    kick = np.zeros((n, 3))
    sel = rng.choice(n, 150, replace=False)
    kick[sel] = u[sel] / b[sel, None]
    out = {}
    for mode in ("cells", "list"):
        with Engine(sys_, precision=prec, neighbour_mode=mode, skin=1.0) as e:
            e.set_particles(xyz, types)
            e.step_with_noise(kick)
            for _ in range(3):
                e.step_with_noise(np.zeros((n, 3)))
            x, _ = e.get_particles()
            m = e.metrics()
        out[mode] = (x, m)
    assert out["list"][1]["neighbour_mode"] == "list"
    assert out["list"][1]["list_builds"] == 1
    same(prec, out["cells"][0], out["list"][0])


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_wide_list_entries_when_offsets_exceed_16_bits(prec):
    """A thin slab of 200,000 particles (4 cell layers of 50,000) whose
    z-neighbour cells lie more than 32767 sorted places apart: the first
    build finds an offset that 16 bits cannot hold and the handle switches to
    32-bit list entries; the trajectory is still the cell walk's (bit for bit
    in FP32C)."""
    rng = np.random.default_rng(4)
    n = 200_000
    sys_ = System([ParticleType("A", 1e6, 1.0)], pair=[PairPotential(A.P2_HARMONIC, [(0, 0)], 10.0, "repulsive")],
                  kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(600, 600, 12), periodic=(1, 1, 1))
    xyz = rng.uniform((0, 0, 0), (600, 600, 12), (n, 3))
    types = np.zeros(n, np.int32)
    xc, _, _ = run(sys_, xyz, types, prec, 60, neighbour_mode="cells")
    xl, _, ml = run(sys_, xyz, types, prec, 60, neighbour_mode="list", skin=1.0)
    assert ml["neighbour_mode"] == "list" and ml["list_entry_bytes"] == 4
    same(prec, xc, xl)


def test_narrow_list_entries_by_default():
    """Config 4's systems (at most 20,000 particles each) keep 16-bit entries."""
    from readdygpu_b200 import configs
    w = configs.config4(n_systems=12, nmin=200, nmax=3000)
    with Engine(w.system, precision="f32c", boxes=w.boxes, neighbour_mode="list", skin=0.6) as e:
        e.set_particles(w.xyz, w.types, offsets=w.offsets)
        e.step(50)
        assert e.metrics()["list_entry_bytes"] == 2
