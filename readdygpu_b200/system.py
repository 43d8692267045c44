"""Host-side description of a ReaDDy system (particle types, potentials, box).

Mirrors the reference's host model (lib/ReaDDyGPU_Cpp/Simulation.hpp:22-181:
ParticleType, DiskPotential, CylinderPotential, SpherePotential, BoxPotential,
HarmonicPotential, ...) and the Java parameter assembly
(src/readdy/impl/assembly/ParticleParametersFactory.java:133-176), and packs
it into the C-ABI struct rdgpu_system_desc.
"""
import ctypes as C
import math

from . import _abi as A

KB_DEFAULT = 0.0083144621  # kJ/(mol K), the value in every reference param_global.xml


class ParticleType:
    """One particle species: D [nm^2/s] and collision radii.

    radius: default collision radius (the pRadius handed to external
    potentials, DiffusionEngine.java:105); radius_with: per-partner-type
    collision radius overrides (param_particles.xml <collisionRadiusMap>).
    """

    def __init__(self, name, D, radius, radius_with=None):
        self.name = name
        self.D = float(D)
        self.radius = float(radius)
        self.radius_with = dict(radius_with or {})


class PairPotential:
    """HARMONIC (subtype attractive/repulsive/spring) or
    WEAK_INTERACTION_PIECEWISE_HARMONIC acting on type pairs."""

    def __init__(self, kind, type_pairs, k, subtype="repulsive", r0=None,
                 length=0.0, depth=0.0):
        self.kind = kind
        self.type_pairs = [tuple(p) for p in type_pairs]
        self.k = float(k)
        self.subtype = subtype
        self.r0 = r0
        self.length = float(length)
        self.depth = float(depth)


class ExternalPotential:
    """DISK, CYLINDER, SPHERE or CUBE acting on particle types."""

    def __init__(self, kind, types, k, subtype="attractive", center=(0, 0, 0),
                 normal=(0, 0, 1), radius=1.0, height=1.0, origin=(0, 0, 0),
                 extension=(1, 1, 1), consider_radius=True):
        self.kind = kind
        self.types = list(types)
        self.k = float(k)
        self.subtype = subtype
        self.center = tuple(float(v) for v in center)
        self.normal = tuple(float(v) for v in normal)
        self.radius = float(radius)
        self.height = float(height)
        self.origin = tuple(float(v) for v in origin)
        self.extension = tuple(float(v) for v in extension)
        self.consider_radius = bool(consider_radius)


class System:
    """Particle types + potentials + box + integrator parameters."""

    def __init__(self, types, pair=(), external=(), kT=None, T=293.15, kB=KB_DEFAULT,
                 dt=1e-9, lo=(0, 0, 0), hi=(1, 1, 1), periodic=(1, 1, 1),
                 max_cutoff=0.0, cell_size=0.0):
        self.types = list(types)
        self.pair = list(pair)
        self.external = list(external)
        self.kB = float(kB)
        self.T = float(kT / kB) if kT is not None else float(T)
        self.dt = float(dt)
        self.lo = tuple(float(v) for v in lo)
        self.hi = tuple(float(v) for v in hi)
        self.periodic = tuple(int(bool(v)) for v in periodic)
        self.max_cutoff = float(max_cutoff)
        self.cell_size = float(cell_size)

    @property
    def n_types(self):
        return len(self.types)

    def box_lengths(self):
        return tuple(h - l for l, h in zip(self.lo, self.hi))

    def volume(self):
        L = self.box_lengths()
        return L[0] * L[1] * L[2]

    def pair_r0(self, i, j):
        """Collision radius sum (ParticleParametersFactory.java:167-170)."""
        ti, tj = self.types[i], self.types[j]
        return ti.radius_with.get(j, ti.radius) + tj.radius_with.get(i, tj.radius)

    def max_pair_cutoff(self):
        m = 0.0
        for p in self.pair:
            for (i, j) in p.type_pairs:
                r0 = p.r0 if p.r0 is not None else self.pair_r0(i, j)
                if p.kind == A.P2_HARMONIC:
                    c = r0 if p.subtype == "repulsive" else self.max_cutoff
                else:
                    c = r0 + p.length
                m = max(m, c)
        return m

    @staticmethod
    def pot_struct(p):
        """A PairPotential as a C rdgpu_pair_pot (type pairs not filled: for bonds)."""
        q = A.PairPot()
        q.kind = p.kind
        q.subtype = A.SUBTYPES[p.subtype] if p.kind == A.P2_HARMONIC else 0
        q.k = p.k
        q.r0 = -1.0 if p.r0 is None else float(p.r0)
        q.length = p.length
        q.depth = p.depth
        return q

    def to_desc(self):
        """Pack into the C struct rdgpu_system_desc."""
        if not 1 <= self.n_types <= A.MAX_TYPES:
            raise ValueError(f"1..{A.MAX_TYPES} particle types supported")
        d = A.SystemDesc()
        d.n_types = self.n_types
        M = A.MAX_TYPES
        for i, t in enumerate(self.types):
            d.D[i] = t.D
            d.p_radius[i] = t.radius
            for j in range(self.n_types):
                d.coll_radius[i * M + j] = t.radius_with.get(j, t.radius)
        if len(self.pair) > A.MAX_PAIR_POTS or len(self.external) > A.MAX_EXT_POTS:
            raise ValueError("too many potentials")
        d.n_pair = len(self.pair)
        for k, p in enumerate(self.pair):
            q = d.pair[k]
            q.kind = p.kind
            q.subtype = A.SUBTYPES[p.subtype] if p.kind == A.P2_HARMONIC else 0
            q.k = p.k
            q.r0 = -1.0 if p.r0 is None else float(p.r0)
            q.length = p.length
            q.depth = p.depth
            for (i, j) in p.type_pairs:
                q.pairs[i * M + j] = 1
                q.pairs[j * M + i] = 1
        d.n_ext = len(self.external)
        for k, e in enumerate(self.external):
            q = d.ext[k]
            q.kind = e.kind
            q.subtype = A.SUBTYPES[e.subtype]
            q.k = e.k
            for a in range(3):
                q.center[a] = e.center[a]
                q.normal[a] = e.normal[a]
                q.origin[a] = e.origin[a]
                q.extension[a] = e.extension[a]
            q.radius = e.radius
            q.height = e.height
            q.consider_radius = int(e.consider_radius)
            for t in e.types:
                q.types[t] = 1
        d.kB, d.T, d.dt = self.kB, self.T, self.dt
        for a in range(3):
            d.lo[a], d.hi[a], d.periodic[a] = self.lo[a], self.hi[a], self.periodic[a]
        d.max_cutoff = self.max_cutoff
        d.cell_size = self.cell_size
        return d


def float_exact_box(L):
    """Nearest box edge that FP32 represents exactly, so the FP32 and the FP64
    engines simulate the same periodic box."""
    import numpy as np
    return float(np.float32(L))


def mobility(system, t):
    """D dt / (kB T) of type t (ParticleParametersFactory.java:155, sign flipped)."""
    return system.types[t].D * system.dt / (system.kB * system.T)


def noise_scale(system, t):
    """sqrt(2 D dt) (ParticleParametersFactory.java:154)."""
    return math.sqrt(2.0 * system.types[t].D * system.dt)
