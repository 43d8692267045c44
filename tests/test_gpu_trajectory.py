"""Config 1 at full size (1,000 particles, 2 species, periodic 50 nm cube,
1,000 steps) run on the engine and on the oracle with the same Philox keys
(seed, step, particle id), compared every 100 steps: positions (minimum
image), potential energy and the MSD per species (D = MSD / 6t).

Bars: FP64 positions within 1e-8 nm, energy and MSD within 1e-8 relative;
FP32C positions within 1e-4 nm, energy within 1e-4 and MSD within 1e-4
relative (FP32 noise transform and FP32 forces against the oracle's FP64).
The trajectories are close enough over 1,000 steps that no statistical bound
is needed; the deviation grows with the contact forces' Lyapunov rate,
which is small for soft harmonic repulsion."""
import numpy as np
import pytest

from readdygpu_b200 import configs

from .test_gpu_parity import Engine, oracle_state

pytestmark = pytest.mark.gpu

SEED = 20261204


def _msd(x0u, xu, types):
    d2 = ((xu - x0u) ** 2).sum(axis=1)
    return [float(d2[types == t].mean()) for t in range(2)]


@pytest.mark.parametrize("prec", ["f64", "f32c"])
@pytest.mark.parametrize("mode", ["cells", "list", "auto"])
def test_config1_full_run_against_oracle(oracle, prec, mode):
    w = configs.config1()
    assert w.n == 1000
    d, _, truth = oracle_state(oracle, w.system, w.xyz, prec)
    L = 50.0
    threads = oracle.max_threads()
    xo = truth.copy()
    xou = truth.copy()                       # oracle trajectory, unwrapped
    tol_x = 1e-8 if prec == "f64" else 1e-4
    tol_r = 1e-8 if prec == "f64" else 1e-4
    devs = []
    with Engine(w.system, precision=prec, seed=SEED, neighbour_mode=mode) as e:
        e.set_particles(w.xyz, w.types)
        if mode == "auto":
            e.autotune()
        for chunk in range(10):
            e.step(100)
            xg, tg = e.get_particles()
            m = e.metrics()
            xn, rc = oracle.run_steps(d, xo, w.types, SEED, chunk * 100, 100, threads)
            assert rc == 0
            step = xn - xo
            step -= L * np.round(step / L)
            xou += step
            xo = xn
            dx = xg - xo
            dx -= L * np.round(dx / L)
            devs.append(float(np.abs(dx).max()))
            assert np.array_equal(tg, w.types)
            assert devs[-1] <= tol_x, (chunk, devs)
            _, Eo = oracle.forces_f64(d, xo, w.types, threads=threads)
            assert abs(m["energy"] - Eo) <= tol_r * abs(Eo), (chunk, m["energy"], Eo)
            mo = _msd(truth, xou, w.types)
            for t in range(2):
                assert abs(m["msd"][t] - mo[t]) <= tol_r * mo[t], (chunk, t, m["msd"][t], mo[t])
        assert m["step"] == 1000
    # D = MSD / (6 t) within a few percent of the input D (1e6, 5e5 nm^2/s):
    # the repulsion barely slows free diffusion at this density
    t_s = 1000 * w.system.dt
    D = [mo[k] / (6 * t_s) for k in range(2)]
    assert abs(D[0] / 1e6 - 1) < 0.1 and abs(D[1] / 5e5 - 1) < 0.1, D
