"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker.  The engine never calls it.
"""
import ctypes as C
import os

import numpy as np

from readdygpu_b200 import _abi as A

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: run `make -C oracle` or __graft_entry__.build()")
        L = C.CDLL(path)
        DP, I32P, U64P, FP = (C.POINTER(C.c_double), C.POINTER(C.c_int32),
                              C.POINTER(C.c_uint64), C.POINTER(C.c_float))
        SD = C.POINTER(A.SystemDesc)
        sig = {
            "orc_pair_gradient": (C.c_int, [C.POINTER(A.PairPot), C.c_double, DP, DP, C.c_double, DP, DP]),
            "orc_ext_gradient": (C.c_int, [C.POINTER(A.ExtPot), C.c_double, DP, DP, DP]),
            "orc_pair_cutoff": (C.c_double, [C.POINTER(A.PairPot), C.c_double, C.c_double]),
            "orc_to_rel_f64": (None, [SD, C.c_int64, DP, DP]),
            "orc_to_rel_f32": (None, [SD, C.c_int64, DP, FP, FP]),
            "orc_forces_f64": (C.c_int, [SD, C.c_int64, DP, I32P, DP, DP, C.c_int]),
            "orc_neighbor_digest_f64": (None, [SD, C.c_int64, DP, I32P, I32P, U64P]),
            "orc_neighbor_digest_f32": (None, [SD, C.c_int64, FP, I32P, I32P, U64P]),
            "orc_step_f64": (C.c_int, [SD, C.c_int64, DP, I32P, DP, C.c_int]),
            "orc_rdf_counts_f64": (None, [SD, C.c_int64, DP, I32P, C.c_int32, C.c_double, U64P]),
            "orc_rdf_counts_f32": (None, [SD, C.c_int64, FP, I32P, C.c_int32, C.c_double, U64P]),
            "orc_rdf_edges2": (None, [C.c_int32, C.c_double, DP]),
            "orc_philox4x32_10": (None, [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
            "orc_bd_normals": (None, [C.c_uint64, C.c_int64, C.c_int64, DP]),
            "orc_splitmix64": (C.c_uint64, [C.c_uint64]),
            "orc_run_steps_f64": (C.c_int, [SD, C.c_int64, DP, I32P, C.c_uint64, C.c_int64, C.c_int64, C.c_int]),
            "orc_max_threads": (C.c_int, []),
            "orc_neighbor_digest_cells_f64": (None, [SD, C.c_int64, DP, I32P, I32P, U64P, C.c_int]),
            "orc_neighbor_digest_cells_f32": (None, [SD, C.c_int64, FP, I32P, I32P, U64P, C.c_int]),
            "orc_rsa_spheres": (C.c_int64, [C.c_int64, C.c_double, C.c_double, C.c_uint64, C.c_int64, DP]),
            "orc_bond_forces_f64": (C.c_int, [SD, C.c_int64, DP, I32P, C.c_int64, I32P, I32P, C.c_int32,
                                              C.POINTER(A.PairPot), DP, DP]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _LIB = L
    return _LIB


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def pair_gradient(pot, r0_pair, x1, x2, dist):
    g = np.zeros(3)
    e = C.c_double()
    x1 = _c(x1, np.float64); x2 = _c(x2, np.float64)
    rc = lib().orc_pair_gradient(C.byref(pot), r0_pair, _p(x1, C.c_double), _p(x2, C.c_double),
                                 dist, _p(g, C.c_double), C.byref(e))
    assert rc == 0
    return g, e.value


def ext_gradient(pot, p_radius, x):
    g = np.zeros(3)
    e = C.c_double()
    x = _c(x, np.float64)
    rc = lib().orc_ext_gradient(C.byref(pot), p_radius, _p(x, C.c_double), _p(g, C.c_double), C.byref(e))
    assert rc == 0
    return g, e.value


def to_rel_f64(desc, xabs):
    xabs = _c(xabs, np.float64)
    n = xabs.size // 3
    out = np.empty_like(xabs)
    lib().orc_to_rel_f64(C.byref(desc), n, _p(xabs, C.c_double), _p(out, C.c_double))
    return out


def to_rel_f32(desc, xabs):
    xabs = _c(xabs, np.float64)
    n = xabs.size // 3
    hi = np.empty(xabs.shape, np.float32)
    comp = np.empty(xabs.shape, np.float32)
    lib().orc_to_rel_f32(C.byref(desc), n, _p(xabs, C.c_double), _p(hi, C.c_float), _p(comp, C.c_float))
    return hi, comp


def forces_f64(desc, xrel, types, threads=1):
    xrel = _c(xrel, np.float64); types = _c(types, np.int32)
    n = types.size
    F = np.zeros((n, 3))
    e = C.c_double()
    lib().orc_forces_f64(C.byref(desc), n, _p(xrel, C.c_double), _p(types, C.c_int32),
                         _p(F, C.c_double), C.byref(e), threads)
    return F, e.value


def bond_forces(desc, xrel, types, ij, pot, pots, F=None, energy=0.0):
    """Adds the forces/energy of bonded pairs (pots: C PairPot structs) to F."""
    xrel = _c(xrel, np.float64); types = _c(types, np.int32)
    ij = _c(ij, np.int32).reshape(-1); pot = _c(pot, np.int32).reshape(-1)
    n = types.size
    F = np.zeros((n, 3)) if F is None else np.ascontiguousarray(F, dtype=np.float64)
    arr = (A.PairPot * max(1, len(pots)))(*pots)
    e = C.c_double(energy)
    rc = lib().orc_bond_forces_f64(C.byref(desc), n, _p(xrel, C.c_double), _p(types, C.c_int32), pot.size,
                                   _p(ij, C.c_int32), _p(pot, C.c_int32), len(pots), arr, _p(F, C.c_double),
                                   C.byref(e))
    if rc:
        raise ValueError("invalid bond")
    return F, e.value


def neighbor_digest(desc, xrel, types, f32=False):
    types = _c(types, np.int32)
    n = types.size
    cnt = np.zeros(n, np.int32)
    h = np.zeros(n, np.uint64)
    if f32:
        x = _c(xrel, np.float32)
        lib().orc_neighbor_digest_f32(C.byref(desc), n, _p(x, C.c_float), _p(types, C.c_int32),
                                      _p(cnt, C.c_int32), _p(h, C.c_uint64))
    else:
        x = _c(xrel, np.float64)
        lib().orc_neighbor_digest_f64(C.byref(desc), n, _p(x, C.c_double), _p(types, C.c_int32),
                                      _p(cnt, C.c_int32), _p(h, C.c_uint64))
    return cnt, h


def neighbor_digest_cells(desc, xrel, types, f32=False, threads=None):
    """neighbor_digest from a cell list with OpenMP (large systems)."""
    types = _c(types, np.int32)
    n = types.size
    cnt = np.zeros(n, np.int32)
    h = np.zeros(n, np.uint64)
    threads = threads or max_threads()
    if f32:
        x = _c(xrel, np.float32)
        lib().orc_neighbor_digest_cells_f32(C.byref(desc), n, _p(x, C.c_float), _p(types, C.c_int32),
                                            _p(cnt, C.c_int32), _p(h, C.c_uint64), threads)
    else:
        x = _c(xrel, np.float64)
        lib().orc_neighbor_digest_cells_f64(C.byref(desc), n, _p(x, C.c_double), _p(types, C.c_int32),
                                            _p(cnt, C.c_int32), _p(h, C.c_uint64), threads)
    return cnt, h


def rsa_spheres(n, L, diam, seed, max_attempts=None):
    """Random sequential insertion (the config-3 input) for the benchmark's
    reference arm; the same coordinates as readdygpu_b200.configs.rsa_spheres."""
    xyz = np.empty((n, 3))
    got = lib().orc_rsa_spheres(n, L, diam, seed, 200 * n if max_attempts is None else max_attempts,
                                _p(xyz, C.c_double))
    if got < n:
        raise RuntimeError(f"random sequential insertion placed only {got} of {n} spheres")
    return xyz


def step_f64(desc, xrel, types, noise, threads=1):
    x = np.array(xrel, dtype=np.float64, copy=True).reshape(-1, 3)
    types = _c(types, np.int32)
    noise = _c(noise, np.float64)
    rc = lib().orc_step_f64(C.byref(desc), types.size, _p(x, C.c_double), _p(types, C.c_int32),
                            _p(noise, C.c_double), threads)
    return x, rc


def rdf_counts(desc, xrel, types, nbins, rmax, f32=False):
    types = _c(types, np.int32)
    S = desc.n_types
    counts = np.zeros(S * S * nbins, np.uint64)
    if f32:
        x = _c(xrel, np.float32)
        lib().orc_rdf_counts_f32(C.byref(desc), types.size, _p(x, C.c_float), _p(types, C.c_int32),
                                 nbins, rmax, _p(counts, C.c_uint64))
    else:
        x = _c(xrel, np.float64)
        lib().orc_rdf_counts_f64(C.byref(desc), types.size, _p(x, C.c_double), _p(types, C.c_int32),
                                 nbins, rmax, _p(counts, C.c_uint64))
    return counts


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)


def bd_normals(seed, step, index):
    o = (C.c_double * 3)()
    lib().orc_bd_normals(seed, step, index, o)
    return list(o)


def bd_normals_many(seed, step, n):
    """bd_normals of indices 0 .. n-1 as an (n, 3) array."""
    out = np.empty((n, 3))
    o = (C.c_double * 3)()
    f = lib().orc_bd_normals
    for i in range(n):
        f(seed, step, i, o)
        out[i] = o
    return out


def splitmix64(x):
    return lib().orc_splitmix64(x)


def run_steps(desc, xrel, types, seed, first_step, nsteps, threads):
    x = np.array(xrel, dtype=np.float64, copy=True).reshape(-1, 3)
    types = _c(types, np.int32)
    rc = lib().orc_run_steps_f64(C.byref(desc), types.size, _p(x, C.c_double), _p(types, C.c_int32),
                                 seed, first_step, nsteps, threads)
    return x, rc


def max_threads():
    return lib().orc_max_threads()
