"""The benchmark workloads: seeded synthetic systems with the shapes, sizes and
distributions of the five benchmark configurations (there is no dataset; the
reference reads its coordinates from tplgy_coordinates.xml).

Units: nm, s, kJ/mol; D in nm^2/s (1e-12 m^2/s = 1e6 nm^2/s);
kB T = 2.437 kJ/mol with kB = 0.0083144621 kJ/(mol K).
Seeds: 20261203 + config index.  Box edges are rounded to FP32-exact values so
that the FP64 and the FP32-compensated engines integrate the same periodic box.
"""
import ctypes as C
import math
import os

import numpy as np

from . import _abi as A
from .system import System, ParticleType, PairPotential, ExternalPotential, KB_DEFAULT, float_exact_box

KT = 2.437
SEED0 = 20261203
_WL = None


def _workloads():
    global _WL
    if _WL is None:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libreaddy_workloads.so")
        _WL = C.CDLL(path)
        _WL.rdgpu_rsa_spheres.restype = C.c_int64
        _WL.rdgpu_rsa_spheres.argtypes = [C.c_int64, C.c_double, C.c_double, C.c_uint64, C.c_int64,
                                          C.POINTER(C.c_double)]
    return _WL


def rsa_spheres(n, L, diam, seed, max_attempts=None):
    """Random sequential insertion without overlap in the periodic box [0,L)^3."""
    xyz = np.empty((n, 3))
    if max_attempts is None:
        max_attempts = 200 * n
    got = _workloads().rdgpu_rsa_spheres(n, L, diam, seed, max_attempts,
                                         xyz.ctypes.data_as(C.POINTER(C.c_double)))
    if got < n:
        raise RuntimeError(f"random sequential insertion placed only {got} of {n} spheres")
    return xyz


def _all_pairs(S):
    return [(i, j) for i in range(S) for j in range(i, S)]


class Workload:
    """A system + its initial particles (+ per-system offsets/boxes for a batch)."""

    def __init__(self, name, system, xyz, types, steps, boxes=None, offsets=None, notes=""):
        self.name = name
        self.system = system
        self.xyz = xyz
        self.types = types
        self.steps = steps
        self.boxes = boxes
        self.offsets = offsets
        self.notes = notes

    @property
    def n(self):
        return int(self.types.size)


def config1(n=1000, steps=1000):
    """1,000 particles of 2 species (500 each), uniform random (overlaps
    allowed) in a periodic 50 nm cube; radii 1.5/2.0 nm; D 1e6/5e5 nm^2/s;
    harmonic repulsion k=10 with cutoff r_i+r_j; kT 2.437; dt 1e-9 s; FP64."""
    rng = np.random.default_rng(SEED0 + 1)
    L = 50.0
    sys_ = System([ParticleType("A", 1e6, 1.5), ParticleType("B", 5e5, 2.0)],
                  pair=[PairPotential(A.P2_HARMONIC, _all_pairs(2), 10.0, "repulsive")],
                  kT=KT, dt=1e-9, lo=(0, 0, 0), hi=(L, L, L), periodic=(1, 1, 1))
    xyz = rng.uniform(0, L, size=(n, 3))
    types = np.repeat(np.arange(2, dtype=np.int32), n // 2)
    types = np.concatenate([types, np.zeros(n - types.size, np.int32)])
    return Workload("config1_plain_1k", sys_, xyz, types, steps)


def config2(n=100_000, steps=10_000):
    """100,000 particles of 4 species in a 400x400x200 nm box periodic in x, y
    (z non-periodic: particles beyond the z bounds are binned into the edge
    cells, no wall); radii 1.0/1.5/2.0/3.0; D log-uniform in [1e5, 1e7] nm^2/s
    per species; harmonic repulsion k=10 for all pairs; piecewise-harmonic
    weak attraction for species 0-1 with depth 2, well r0 = 1.1(r0+r1),
    width l = 0.4(r0+r1) (cutoff 1.5(r0+r1)) and inner k = 10; attractive
    disk at z=0, normal z, radius 150, k=10 on species 3."""
    rng = np.random.default_rng(SEED0 + 2)
    radii = [1.0, 1.5, 2.0, 3.0]
    D = [float(v) for v in 10 ** rng.uniform(5, 7, size=4)]
    types_ = [ParticleType(f"S{i}", D[i], radii[i]) for i in range(4)]
    s01 = radii[0] + radii[1]
    pair = [PairPotential(A.P2_HARMONIC, _all_pairs(4), 10.0, "repulsive"),
            PairPotential(A.P2_WEAK_PIECEWISE, [(0, 1)], 10.0, r0=1.1 * s01, length=0.4 * s01, depth=2.0)]
    ext = [ExternalPotential(A.P1_DISK, [3], 10.0, "attractive", center=(0, 0, 0), normal=(0, 0, 1), radius=150.0)]
    sys_ = System(types_, pair=pair, external=ext, kT=KT, dt=1e-9,
                  lo=(-200, -200, -100), hi=(200, 200, 100), periodic=(1, 1, 0))
    xyz = np.empty((n, 3))
    xyz[:, 0] = rng.uniform(-200, 200, n)
    xyz[:, 1] = rng.uniform(-200, 200, n)
    xyz[:, 2] = rng.uniform(-100, 100, n)
    types = (np.arange(n) * 4 // n).astype(np.int32)
    return Workload("config2_4species_100k", sys_, xyz, types, steps)


def config3(n=1_000_000, steps=5_000, phi=0.30, rsa=None):
    """n identical spheres of radius 2 nm at volume fraction phi in a periodic
    cube (seeded random sequential insertion without overlap); D 1e6 nm^2/s;
    harmonic repulsion k=10 (cutoff 4 nm = cell size); RDF 200 bins over
    0-20 nm every 100 steps.  rsa: the insertion routine (default
    rsa_spheres; any routine with its arguments and coordinates)."""
    r = 2.0
    L = float_exact_box((n * 4.0 / 3.0 * math.pi * r ** 3 / phi) ** (1.0 / 3.0))
    sys_ = System([ParticleType("A", 1e6, r)],
                  pair=[PairPotential(A.P2_HARMONIC, [(0, 0)], 10.0, "repulsive")],
                  kT=KT, dt=1e-9, lo=(0, 0, 0), hi=(L, L, L), periodic=(1, 1, 1), cell_size=4.0)
    xyz = (rsa or rsa_spheres)(n, L, 2 * r, SEED0 + 3)
    return Workload(f"config3_rsa_{n}", sys_, xyz, np.zeros(n, np.int32), steps,
                    notes="RDF 200 bins 0-20 nm every 100 steps")


def config4(n_systems=512, steps=2_000, nmin=500, nmax=20_000):
    """n_systems independent periodic cubes, N_k log-uniform in [nmin, nmax],
    volume fraction U(0.1, 0.3), 2 species 50/50 with radii 1.5/2.0 and
    D 1e6/5e5 nm^2/s (the config-1 species), harmonic repulsion k=10,
    uniform random positions (overlaps allowed), own Philox seed each."""
    rng = np.random.default_rng(SEED0 + 4)
    Ns = np.rint(np.exp(rng.uniform(math.log(nmin), math.log(nmax), n_systems))).astype(np.int64)
    phis = rng.uniform(0.1, 0.3, n_systems)
    vbar = 4.0 / 3.0 * math.pi * (1.5 ** 3 + 2.0 ** 3) / 2.0
    sys_ = System([ParticleType("A", 1e6, 1.5), ParticleType("B", 5e5, 2.0)],
                  pair=[PairPotential(A.P2_HARMONIC, _all_pairs(2), 10.0, "repulsive")],
                  kT=KT, dt=1e-9, lo=(0, 0, 0), hi=(1, 1, 1), periodic=(1, 1, 1))
    boxes, xs, ts = [], [], []
    for k in range(n_systems):
        L = float_exact_box((Ns[k] * vbar / phis[k]) ** (1.0 / 3.0))
        boxes.append(((0.0, 0.0, 0.0), (L, L, L), (1, 1, 1), SEED0 + 4 + 1000 * (k + 1)))
        xs.append(rng.uniform(0, L, size=(Ns[k], 3)))
        t = np.zeros(Ns[k], np.int32)
        t[Ns[k] // 2:] = 1
        ts.append(t)
    offsets = np.concatenate([[0], np.cumsum(Ns)]).astype(np.int64)
    return Workload(f"config4_batch_{n_systems}", sys_, np.concatenate(xs), np.concatenate(ts), steps,
                    boxes=boxes, offsets=offsets)


def config5(n=250_000, steps=1_000_000, n_shell=15_000):
    """n particles of 3 species in a spherical vesicle of radius 120 nm
    (non-periodic box +-130 nm); radii 1.0 nm each; species 0/1 inside
    (SPHERE attractive, k=10), species 2 on the shell (SPHERE membrane, k=10);
    harmonic repulsion k=10 for all pairs; piecewise weak attraction between
    species 1 and 2 (depth 2, r0 = 1.1 sigma, l = 0.4 sigma); D 1e6 nm^2/s."""
    rng = np.random.default_rng(SEED0 + 5)
    R = 120.0
    rad = 1.0
    types_ = [ParticleType(f"S{i}", 1e6, rad) for i in range(3)]
    sig = 2 * rad
    pair = [PairPotential(A.P2_HARMONIC, _all_pairs(3), 10.0, "repulsive"),
            PairPotential(A.P2_WEAK_PIECEWISE, [(1, 2)], 10.0, r0=1.1 * sig, length=0.4 * sig, depth=2.0)]
    ext = [ExternalPotential(A.P1_SPHERE, [0, 1], 10.0, "attractive", center=(0, 0, 0), radius=R),
           ExternalPotential(A.P1_SPHERE, [2], 10.0, "membrane", center=(0, 0, 0), radius=R)]
    sys_ = System(types_, pair=pair, external=ext, kT=KT, dt=1e-9,
                  lo=(-130, -130, -130), hi=(130, 130, 130), periodic=(0, 0, 0))
    n_in = n - n_shell
    u = rng.normal(size=(n_in, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    rr = (R - rad) * rng.uniform(0, 1, n_in) ** (1.0 / 3.0)
    inside = u * rr[:, None]
    v = rng.normal(size=(n_shell, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    shell = v * R
    xyz = np.concatenate([inside, shell])
    types = np.concatenate([np.arange(n_in) % 2, np.full(n_shell, 2)]).astype(np.int32)
    return Workload(f"config5_vesicle_{n}", sys_, xyz, types, steps)


CONFIGS = {1: config1, 2: config2, 3: config3, 4: config4, 5: config5}
