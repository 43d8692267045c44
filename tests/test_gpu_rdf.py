"""RDF counts of the engine (rdgpu_rdf through the C ABI) against the oracle,
bit-exact, on the cases that stress the RDF grid: a periodic axis with
exactly 5 cells of edge rmax/2 (the fewest the row kernel takes), an open
axis, particles on cell faces and on the periodic bounds, pairs at exactly a
bin edge and at exactly rmax, coincident particles, three species, a batch of
boxes of different sizes, and a histogram too large for shared memory.
Counts are of ordered pairs (both orientations of every pair within rmax,
CudaSimulation.cu:1815-1818)."""
import numpy as np
import pytest

from readdygpu_b200 import _abi as A
from readdygpu_b200.system import System, ParticleType, PairPotential, float_exact_box

from .test_gpu_parity import Engine, oracle_state

pytestmark = pytest.mark.gpu
PRECS = ["f64", "f32c"]


def edge_box_system(rmax, n=2500, seed=3):
    """A box with 5 cells of edge >= rmax/2 along x (periodic), 7 along y
    (periodic) and an open z; random particles plus planted structure."""
    Lx = float_exact_box(5.0 * 0.5 * rmax * (1.0 + 3e-5))
    Ly = float_exact_box(7.3 * 0.5 * rmax)
    Lz = 3.2 * rmax
    types = [ParticleType(f"T{i}", 1e6, 1.0 + 0.25 * i) for i in range(3)]
    sys_ = System(types, pair=[PairPotential(A.P2_HARMONIC, [(0, 0), (1, 2)], 10.0, "repulsive")],
                  kT=2.437, dt=1e-9, lo=(0, 0, -0.5 * Lz), hi=(Lx, Ly, 0.5 * Lz), periodic=(1, 1, 0))
    rng = np.random.default_rng(seed)
    xyz = [np.column_stack([rng.uniform(0, Lx, n), rng.uniform(0, Ly, n), rng.uniform(-0.5 * Lz, 0.5 * Lz, n)])]
    w = rmax / 40.0
    c = 0.5 * rmax
    base = np.array([0.25 * Lx, 0.5 * Ly, 0.0])
    planted = []
    for k in (1, 7, 20, 39, 40):                        # exactly on bin edges, and exactly rmax
        planted += [base, base + np.array([k * w, 0, 0])]
    planted += [np.array([0.0, 1.0, 0.0]), np.array([Lx - 0.3 * rmax, 1.0, 0.0])]   # across the x bound
    planted += [np.array([c, c, 0.0]), np.array([c, c + 0.99 * rmax, 0.0])]       # on cell faces
    planted += [np.array([2 * c, 3 * c, 0.1]), np.array([2 * c, 3 * c, 0.1])]     # coincident
    planted += [np.array([1.0, 2.0, 0.5 * Lz - 1e-3]), np.array([1.0, 2.0, 0.5 * Lz + 0.4 * rmax])]  # past the open bound
    xyz.append(np.array(planted))
    xyz = np.concatenate(xyz)
    tt = rng.integers(0, 3, xyz.shape[0]).astype(np.int32)
    return sys_, xyz, tt


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("mode", ["cells", "list"])
def test_rdf_five_cells_open_axis_planted_pairs(oracle, prec, mode):
    rmax, nbins = 8.0, 40
    sys_, xyz, types = edge_box_system(rmax)
    d, stored, _ = oracle_state(oracle, sys_, xyz, prec)
    with Engine(sys_, precision=prec, neighbour_mode=mode, skin=0.5) as e:
        e.set_particles(xyz, types)
        c, _ = e.rdf(nbins, rmax, accumulate=False)
        c2, _ = e.rdf(nbins, rmax, accumulate=False)
    co = oracle.rdf_counts(d, stored, types, nbins, rmax, f32=(prec == "f32c"))
    assert c.sum() > 1000
    assert np.array_equal(c.ravel(), co)
    assert np.array_equal(c2, c)
    assert np.array_equal(c, c.transpose(1, 0, 2))


@pytest.mark.parametrize("prec", PRECS)
def test_rdf_batch_of_boxes_equals_sum_over_systems(oracle, prec):
    """A batch of periodic cubes of different sizes (10 to 27 RDF cells per
    edge): the batch's counts are the sum of the oracle's counts of every
    box."""
    from readdygpu_b200 import configs
    w = configs.config4(n_systems=12, nmin=300, nmax=6000)
    rmax, nbins = 7.0, 70
    with Engine(w.system, precision=prec, boxes=w.boxes) as e:
        e.set_particles(w.xyz, w.types, offsets=w.offsets)
        c, _ = e.rdf(nbins, rmax, accumulate=False)
    total = np.zeros(c.size, np.uint64)
    for k, (lo, hi, per, _) in enumerate(w.boxes):
        d = w.system.to_desc()
        for a in range(3):
            d.lo[a], d.hi[a], d.periodic[a] = lo[a], hi[a], int(per[a])
        sl = slice(int(w.offsets[k]), int(w.offsets[k + 1]))
        if prec == "f64":
            stored = oracle.to_rel_f64(d, w.xyz[sl]).reshape(-1, 3)
        else:
            stored = oracle.to_rel_f32(d, w.xyz[sl])[0].reshape(-1, 3)
        total += oracle.rdf_counts(d, stored, w.types[sl], nbins, rmax, f32=(prec == "f32c"))
    assert total.sum() > 0
    assert np.array_equal(c.ravel(), total)


@pytest.mark.parametrize("prec", PRECS)
def test_rdf_histogram_larger_than_shared_memory(oracle, prec):
    """3000 bins: the block histogram does not fit next to the edge table, so
    the row kernel counts into global memory."""
    from readdygpu_b200 import configs
    w = configs.config1(n=1500)
    sys_, xyz, types = w.system, w.xyz, w.types
    rmax, nbins = 18.0, 3000
    d, stored, _ = oracle_state(oracle, sys_, xyz, prec)
    with Engine(sys_, precision=prec) as e:
        e.set_particles(xyz, types)
        c, _ = e.rdf(nbins, rmax, accumulate=False)
    co = oracle.rdf_counts(d, stored, types, nbins, rmax, f32=(prec == "f32c"))
    assert co.sum() > 0
    assert np.array_equal(c.ravel(), co)


@pytest.mark.parametrize("prec", PRECS)
@pytest.mark.parametrize("species", [1, 2])
def test_rdf_lattice_pairs_on_bin_edges(oracle, prec, species):
    """A simple cubic lattice of spacing 1 nm with bins of 0.1 nm: every pair
    distance is sqrt(n) nm, and those with n a perfect square lie exactly on
    a bin edge in real arithmetic (the FP64 edge table rounds them to one side
    or the other); with two species, the second, shifted by a quarter
    spacing, adds distances off the lattice.  Counts bit-exact."""
    n = 18
    g = np.arange(n, dtype=np.float64)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    lat = np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])
    if species == 1:
        xyz, types = lat, np.zeros(len(lat), np.int32)
    else:
        xyz = np.concatenate([lat, lat[::3] + 0.25])
        types = np.concatenate([np.zeros(len(lat), np.int32), np.ones(len(lat[::3]), np.int32)])
    t = [ParticleType("A", 1e6, 0.3), ParticleType("B", 1e6, 0.3)][:species]
    sys_ = System(t, pair=[PairPotential(A.P2_HARMONIC, [(0, 0)], 10.0, "repulsive")],
                  kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(float(n), float(n), float(n)), periodic=(1, 1, 1))
    rmax, nbins = 7.0, 70
    d, stored, _ = oracle_state(oracle, sys_, xyz, prec)
    with Engine(sys_, precision=prec, neighbour_mode="cells") as e:
        e.set_particles(xyz, types)
        c, _ = e.rdf(nbins, rmax, accumulate=False)
    co = oracle.rdf_counts(d, stored, types, nbins, rmax, f32=(prec == "f32c"))
    assert co.sum() > 0
    assert np.array_equal(c.ravel(), co)


@pytest.mark.parametrize("prec", PRECS)
def test_rdf_dense_cluster_many_passes(oracle, prec):
    """600 particles packed into one RDF cell (3 nm cube) among 1,000 spread
    over the box: the cluster's cell holds ten passes of own particles, its
    candidate queue fills and drains many times, and the own cell's pairs
    span passes.  Three species; counts bit-exact."""
    rng = np.random.default_rng(21)
    L = 40.0
    types_ = [ParticleType(f"T{i}", 1e6, 0.5) for i in range(3)]
    sys_ = System(types_, pair=[PairPotential(A.P2_HARMONIC, [(0, 0)], 10.0, "repulsive")],
                  kT=2.437, dt=1e-9, lo=(0, 0, 0), hi=(L, L, L), periodic=(1, 1, 1))
    cluster = rng.uniform(13.6, 16.6, size=(600, 3))     # inside RDF cell 3 of edge 40/9 nm per axis
    spread = rng.uniform(0, L, size=(1000, 3))
    xyz = np.concatenate([cluster, spread])
    types = rng.integers(0, 3, len(xyz)).astype(np.int32)
    rmax, nbins = 8.0, 64
    d, stored, _ = oracle_state(oracle, sys_, xyz, prec)
    with Engine(sys_, precision=prec, neighbour_mode="cells") as e:
        e.set_particles(xyz, types)
        c, _ = e.rdf(nbins, rmax, accumulate=False)
    co = oracle.rdf_counts(d, stored, types, nbins, rmax, f32=(prec == "f32c"))
    assert co.sum() > 600 * 599
    assert np.array_equal(c.ravel(), co)
