"""Python handle over the C ABI (include/readdy_b200.h).

Mirrors the operations of the reference's CudaSimulation host wrapper
(lib/ReaDDyGPU_Cpp/CudaKernels/CudaSimulation.cuh:39-116): initialize ->
Engine(...), copyPosToDevice/createNeighborList -> set_particles,
simulate -> step, copyPosFromDevice -> get_particles, callRDFCalculation/
copyRDFMatrix -> rdf.  Errors raise RdgpuError with the library's message
(the reference returns 1 and prints, CudaSimulation.cu:138-455).
"""
import ctypes as C

import numpy as np

from . import _abi as A


class RdgpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"rdgpu error {code}: {msg}")
        self.code = code


def _lib():
    from . import load
    return load()


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Engine:
    """One handle: a single system, or a batch of systems sharing types and
    potentials (boxes=[(lo, hi, periodic, seed), ...])."""

    NB_MODES = {"auto": A.NB_AUTO, "cells": A.NB_CELLS, "list": A.NB_LIST}

    def __init__(self, system, precision="f64", device=0, seed=0, boxes=None, neighbour_mode="auto",
                 skin=0.0, graph_steps=0):
        self.system = system
        self._desc = system.to_desc()
        opt = A.Options()
        opt.precision = {"f64": A.PREC_F64, "f32c": A.PREC_F32C}[precision]
        opt.device = device
        opt.neighbour_mode = self.NB_MODES[neighbour_mode]
        opt.skin = skin
        opt.graph_steps = graph_steps
        opt.seed = seed
        self.precision = precision
        h = C.c_void_p()
        L = _lib()
        if boxes is None:
            rc = L.rdgpu_create(C.byref(self._desc), C.byref(opt), C.byref(h))
            self.n_systems = 1
        else:
            arr = (A.Box * len(boxes))()
            for k, (lo, hi, per, sd) in enumerate(boxes):
                for a in range(3):
                    arr[k].lo[a], arr[k].hi[a], arr[k].periodic[a] = lo[a], hi[a], int(per[a])
                arr[k].seed = sd
            rc = L.rdgpu_create_batch(C.byref(self._desc), len(boxes), arr, C.byref(opt), C.byref(h))
            self.n_systems = len(boxes)
        if rc != 0:
            raise RdgpuError(rc, L.rdgpu_last_error(None).decode())
        self._h = h
        self.n = 0

    # -- plumbing --------------------------------------------------------
    def _check(self, rc):
        if rc != 0:
            raise RdgpuError(rc, _lib().rdgpu_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            _lib().rdgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def stream(self):
        return _lib().rdgpu_stream(self._h)

    def launch_count(self):
        return _lib().rdgpu_launch_count(self._h)

    def autotune(self):
        """Run the neighbour-search autotuner now (neighbour_mode="auto")."""
        self._check(_lib().rdgpu_autotune(self._h))

    def step_profile(self, nsteps):
        """Mean ms per step of the fused step kernel and of the counting sort."""
        ks, ss = C.c_double(), C.c_double()
        self._check(_lib().rdgpu_step_profile(self._h, int(nsteps), C.byref(ks), C.byref(ss)))
        return ks.value, ss.value

    # -- state -----------------------------------------------------------
    def set_particles(self, xyz, types, offsets=None):
        """Upload positions (n, 3) and types; float32 positions go through
        rdgpu_set_particles_f32 (half the bytes), anything else as float64."""
        f32 = isinstance(xyz, np.ndarray) and xyz.dtype == np.float32
        xyz = np.ascontiguousarray(xyz, dtype=np.float32 if f32 else np.float64).reshape(-1, 3)
        types = np.ascontiguousarray(types, dtype=np.int32).reshape(-1)
        n = types.size
        if offsets is not None:
            off = np.ascontiguousarray(offsets, dtype=np.int64)
            offp = _p(off, C.c_int64)
        else:
            offp = None
        if f32:
            rc = _lib().rdgpu_set_particles_f32(self._h, offp, n, _p(xyz, C.c_float), _p(types, C.c_int32))
        else:
            rc = _lib().rdgpu_set_particles(self._h, offp, n, _p(xyz, C.c_double), _p(types, C.c_int32))
        self._check(rc)
        self.n = n

    def get_particles(self, xyz=None, types=None):
        """Positions (n, 3) float64 and types; into the given C-contiguous
        arrays when passed (e.g. pinned host buffers); a float32 xyz array
        is filled through rdgpu_get_particles_f32."""
        if xyz is None:
            xyz = np.empty((self.n, 3))
        if types is None:
            types = np.empty(self.n, np.int32)
        assert xyz.dtype in (np.float64, np.float32) and xyz.shape == (self.n, 3) and xyz.flags.c_contiguous
        assert types.dtype == np.int32 and types.shape == (self.n,) and types.flags.c_contiguous
        if xyz.dtype == np.float32:
            rc = _lib().rdgpu_get_particles_f32(self._h, _p(xyz, C.c_float), _p(types, C.c_int32))
        else:
            rc = _lib().rdgpu_get_particles(self._h, _p(xyz, C.c_double), _p(types, C.c_int32))
        self._check(rc)
        return xyz, types

    def set_bonds(self, ij, pot, potentials):
        """Bonded pairs of particle groups: ij (n, 2) particle indices, pot (n,)
        indices into potentials (PairPotential, type pairs ignored)."""
        from .system import System
        ij = np.ascontiguousarray(ij, dtype=np.int32).reshape(-1, 2)
        pot = np.ascontiguousarray(pot, dtype=np.int32).reshape(-1)
        arr = (A.PairPot * max(1, len(potentials)))()
        for k, p in enumerate(potentials):
            arr[k] = System.pot_struct(p)
        self._check(_lib().rdgpu_set_bonds(self._h, ij.shape[0], _p(ij, C.c_int32), _p(pot, C.c_int32),
                                           len(potentials), C.cast(arr, C.c_void_p)))

    def apply_edits(self, edits):
        """Reaction edits in the layout of ReaDDy's cReactions entries:
        rows of (readdyId, newType, x, y, z, gpuIndex)."""
        e = np.ascontiguousarray(edits, dtype=np.float32).reshape(-1, 6)
        self._check(_lib().rdgpu_apply_edits(self._h, _p(e, C.c_float), e.shape[0]))
        n = C.c_int64()
        _lib().rdgpu_num_particles(self._h, C.byref(n))
        self.n = n.value

    # -- dynamics --------------------------------------------------------
    def step(self, nsteps=1):
        self._check(_lib().rdgpu_step(self._h, int(nsteps)))

    def step_with_noise(self, noise):
        noise = np.ascontiguousarray(noise, dtype=np.float64).reshape(-1)
        assert noise.size == 3 * self.n
        self._check(_lib().rdgpu_step_with_noise(self._h, _p(noise, C.c_double)))

    def set_seed(self, seed, sys=0):
        self._check(_lib().rdgpu_set_seed(self._h, sys, seed))

    # -- observables -----------------------------------------------------
    def forces(self):
        F = np.empty((self.n, 3))
        e = C.c_double()
        self._check(_lib().rdgpu_forces(self._h, _p(F, C.c_double), C.byref(e)))
        return F, e.value

    def neighbor_digest(self):
        cnt = np.empty(self.n, np.int32)
        h = np.empty(self.n, np.uint64)
        self._check(_lib().rdgpu_neighbor_digest(self._h, _p(cnt, C.c_int32), _p(h, C.c_uint64)))
        return cnt, h

    def debug_noise(self, step):
        out = np.empty((self.n, 3))
        self._check(_lib().rdgpu_debug_noise(self._h, int(step), _p(out, C.c_double)))
        return out

    def rdf(self, nbins, rmax, accumulate=True):
        S = self.system.n_types
        out = np.empty(S * S * nbins, np.uint64)
        fr = C.c_int64()
        self._check(_lib().rdgpu_rdf(self._h, nbins, rmax, int(accumulate), _p(out, C.c_uint64), C.byref(fr)))
        return out.reshape(S, S, nbins), fr.value

    def rdf_normalized(self, nbins):
        S = self.system.n_types
        g = np.empty(S * S * nbins)
        self._check(_lib().rdgpu_rdf_normalized(self._h, _p(g, C.c_double)))
        return g.reshape(S, S, nbins)

    def metrics(self):
        m = A.Metrics()
        self._check(_lib().rdgpu_metrics_get(self._h, C.byref(m)))
        S = self.system.n_types
        return {"energy": m.energy, "msd": list(m.msd[:S]), "count": list(m.count[:S]),
                "step": m.step, "neighbour_mode": {A.NB_CELLS: "cells", A.NB_LIST: "list"}.get(m.neighbour_mode),
                "list_builds": m.list_builds, "skin": m.skin, "list_capacity": m.list_capacity,
                "list_entry_bytes": m.list_entry_bytes}
