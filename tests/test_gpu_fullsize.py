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
