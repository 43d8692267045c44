"""FP32 coordinate transfers (rdgpu_set_particles_f32 / rdgpu_get_particles_f32,
the reference's float frames) against the FP64 calls."""
import numpy as np
import pytest

from .test_gpu_parity import Engine, cfg1

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", ["f32c", "f64"])
def test_f32_upload_equals_f64_upload_of_the_same_values(prec):
    sys_, xyz, types = cfg1(1500)
    x32 = xyz.astype(np.float32)
    out = []
    for use_f32 in (False, True):
        with Engine(sys_, precision=prec, seed=6) as e:
            e.set_particles(x32 if use_f32 else x32.astype(np.float64), types)
            x0, t0 = e.get_particles()
            e.step(60)
            x1, t1 = e.get_particles()
            f1 = np.empty((e.n, 3), np.float32)
            e.get_particles(f1, np.empty(e.n, np.int32))
            out.append((x0, t0, x1, t1, f1))
    # the uploads are identical; after steps FP32C is bit-reproducible, FP64
    # only to rounding (the order within a cell, hence of the FP64 pair sums,
    # follows the counting sort's atomics)
    for q, (a, b) in enumerate(zip(out[0], out[1])):
        if prec == "f64" and q in (2, 4):
            assert np.abs(a - b).max() <= 1e-9
        else:
            np.testing.assert_array_equal(a, b)
    x0, t0, x1, t1, f1 = out[1]
    np.testing.assert_array_equal(x0, x32.astype(np.float64))     # exact upload
    np.testing.assert_array_equal(t0, types)
    np.testing.assert_array_equal(f1, x1.astype(np.float32))      # download rounds to FP32


def test_f32_transfers_of_a_batch():
    from readdygpu_b200 import configs
    w = configs.config4(n_systems=6, nmin=200, nmax=1500)
    x32 = w.xyz.astype(np.float32)
    with Engine(w.system, precision="f32c", boxes=w.boxes) as e:
        e.set_particles(x32, w.types, offsets=w.offsets)
        f = np.empty((e.n, 3), np.float32)
        t = np.empty(e.n, np.int32)
        e.get_particles(f, t)
        np.testing.assert_array_equal(f, x32)
        np.testing.assert_array_equal(t, w.types)
        e.step(30)
        x, _ = e.get_particles()
        e.get_particles(f, t)
        np.testing.assert_array_equal(f, x.astype(np.float32))
