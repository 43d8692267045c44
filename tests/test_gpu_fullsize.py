"""The benchmark configurations at their full sizes, through properties that do
not need a small case: RDF counts of config 3 (1,000,000 RSA spheres, 200 bins
over 0-20 nm) bit-exact against the oracle's (OpenMP) counts in both
precisions and both neighbour modes, and the FP32C force error against FP64
for configs 2 (100,000), 4 (2,445,685) and 5 (250,000)."""
import numpy as np
import pytest

from readdygpu_b200 import configs, precision

from .test_gpu_parity import Engine, oracle_state

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def config3_full():
    return configs.config3()


@pytest.mark.parametrize("prec", ["f64", "f32c"])
def test_config3_rdf_full_size_bit_exact(oracle, config3_full, prec):
    w = config3_full
    assert w.n == 1_000_000
    d, stored, _ = oracle_state(oracle, w.system, w.xyz, prec)
    co = oracle.rdf_counts(d, stored, w.types, 200, 20.0, f32=(prec == "f32c"))
    for mode in ("cells", "list"):
        with Engine(w.system, precision=prec, neighbour_mode=mode, skin=1.0) as e:
            e.set_particles(w.xyz, w.types)
            c, _ = e.rdf(200, 20.0, accumulate=False)
        assert np.array_equal(c.reshape(-1), co), (mode, np.abs(c.reshape(-1).astype(np.int64) - co.astype(np.int64)).max())
    assert co.sum() > 0
    if prec == "f64":
        # RSA without overlap: no pair closer than 2 radii (4 nm = bin 40);
        # FP32 rounding may move near-contact pairs into bin 39
        assert co[:40].sum() == 0


@pytest.mark.parametrize("cfg", [2, 4, 5])
def test_fp32c_force_error_full_size(cfg):
    w = configs.CONFIGS[cfg]()
    r = precision.force_error(w)
    assert r["force_rel_err"] <= 1e-5, r
    assert r["energy_rel_err"] <= 1e-5, r


def _per_system(w):
    """(descriptor, particle slice) of every system of a workload."""
    if w.boxes is None:
        return [(w.system.to_desc(), slice(0, w.n))]
    out = []
    for k, (lo, hi, per, _) in enumerate(w.boxes):
        d = w.system.to_desc()
        for a in range(3):
            d.lo[a], d.hi[a], d.periodic[a] = lo[a], hi[a], int(per[a])
        out.append((d, slice(int(w.offsets[k]), int(w.offsets[k + 1]))))
    return out


def _stored(O, d, xyz, prec):
    """The positions as the engine stores them (box-relative; FP32 for FP32C)."""
    if prec == "f64":
        return O.to_rel_f64(d, xyz).reshape(-1, 3)
    hi, _ = O.to_rel_f32(d, xyz)
    return hi.reshape(-1, 3)


FULL = {2: configs.config2, 4: configs.config4, 5: configs.config5}


@pytest.mark.parametrize("prec", ["f64", "f32c"])
@pytest.mark.parametrize("cfg", [2, 4, 5])
def test_full_size_neighbours_and_forces_against_oracle(oracle, cfg, prec):
    """Configs 2 (100,000, z open, weak interaction + disk), 4 (512 systems,
    2,445,685 particles) and 5 (250,000, sphere + membrane) at full size,
    engine against the oracle on the same stored positions:
      * neighbour sets (count and hash of partner ids per particle): bit-exact,
        with the FP64 and the FP32 predicate;
      * FP64 forces ||dF||/||F|| <= 1e-12, energy 1e-10 relative;
      * FP32C forces ||dF||/||F|| <= 1e-5, per particle 1e-4 max(|F_i|, F_rms),
        energy 1e-5 relative."""
    w = FULL[cfg]()
    kw = {"boxes": w.boxes} if w.boxes is not None else {}
    with Engine(w.system, precision=prec, **kw) as e:
        e.set_particles(w.xyz, w.types, offsets=w.offsets)
        cnt, h = e.neighbor_digest()
        F, E = e.forces()
    threads = oracle.max_threads()
    Fo = np.zeros_like(F)
    Eo = 0.0
    for d, sl in _per_system(w):
        x = _stored(oracle, d, w.xyz[sl], prec)
        oc, oh = oracle.neighbor_digest_cells(d, x, w.types[sl], f32=(prec == "f32c"), threads=threads)
        assert np.array_equal(cnt[sl], oc), (cfg, prec, "counts", int(np.abs(cnt[sl] - oc).max()))
        assert np.array_equal(h[sl], oh), (cfg, prec, "hashes")
        Fo[sl], e_ = oracle.forces_f64(d, x.astype(np.float64), w.types[sl], threads=threads)
        Eo += e_
    assert cnt.sum() > 0
    rel = np.linalg.norm(F - Fo) / np.linalg.norm(Fo)
    if prec == "f64":
        assert rel <= 1e-12, rel
        assert abs(E - Eo) <= 1e-10 * max(1.0, abs(Eo)), (E, Eo)
    else:
        assert rel <= 1e-5, rel
        per = np.linalg.norm(F - Fo, axis=1)
        mag = np.linalg.norm(Fo, axis=1)
        rms = np.sqrt(np.mean(mag ** 2))
        assert np.all(per <= 1e-4 * np.maximum(mag, rms)), (per / np.maximum(mag, rms)).max()
        assert abs(E - Eo) <= 1e-5 * max(1.0, abs(Eo)), (E, Eo)


@pytest.mark.parametrize("mode", ["cells", "list"])
def test_config3_rdf_frames_over_a_run(oracle, mode):
    """Config 3's RDF (200 bins over 0-20 nm) at every 100th step of a
    1,000-step FP64 run on 100,000 RSA spheres: each frame's counts equal the
    oracle's counts of the positions the engine holds at that step, bit for
    bit.  (FP64 only: the FP32C engine bins its stored FP32 coordinates,
    which a download returns compensated; its frames are checked at upload
    in test_config3_rdf_full_size_bit_exact.)"""
    w = configs.config3(n=100_000)
    d = w.system.to_desc()
    with Engine(w.system, precision="f64", seed=9, neighbour_mode=mode, skin=1.0) as e:
        e.set_particles(w.xyz, w.types)
        for frame in range(10):
            e.step(100)
            c, _ = e.rdf(200, 20.0, accumulate=False)
            x, _ = e.get_particles()
            co = oracle.rdf_counts(d, oracle.to_rel_f64(d, x).reshape(-1, 3), w.types, 200, 20.0)
            assert np.array_equal(c.reshape(-1), co), (frame, int(np.abs(c.reshape(-1).astype(np.int64) - co.astype(np.int64)).max()))
        assert e.metrics()["step"] == 1000
