"""Short rdgpu_step calls replay captured graphs (the remainder below the
100-step graph as powers of two): the same trajectory bit for bit whatever
the split of the steps into calls, and two kernel launches per pair-list step
(step kernel + list check) plus the re-sorts."""
import numpy as np
import pytest

from readdygpu_b200 import configs

from .test_gpu_parity import Engine

pytestmark = pytest.mark.gpu

SPLITS = ([100], [20] * 5, [7, 13, 64, 16], [1] * 3 + [97])


@pytest.mark.parametrize("mode", ["cells", "list"])
def test_short_calls_are_graphed_and_identical(mode):
    w = configs.config4(n_systems=16, nmin=300, nmax=3000)
    out = []
    for split in SPLITS:
        with Engine(w.system, precision="f32c", boxes=w.boxes, neighbour_mode=mode, skin=0.8) as e:
            e.set_particles(w.xyz, w.types, offsets=w.offsets)
            e.autotune()                      # captures the graphs: no call below captures
            # metrics() evaluates the energy on fresh cells (one re-sort and
            # build, counted in both figures)
            l0 = e.launch_count()
            b0 = e.metrics()["list_builds"]
            for n in split:
                e.step(n)
            launches = e.launch_count() - l0
            m = e.metrics()
            out.append(e.get_particles()[0])
        assert m["step"] == 100
        graphs = sum(bin(n % 100).count("1") + n // 100 for n in split)
        if mode == "list":
            assert launches == 2 * 100 + graphs + 6 * (m["list_builds"] - b0), (split, launches)
        else:
            assert launches == 4 * 100 + graphs, (split, launches)
    for x in out[1:]:
        assert np.array_equal(out[0], x)


def test_retune_after_list_overflow_keeps_the_trajectory():
    """An AUTO handle whose lists outgrow their capacity while stepping (config
    2's weak attraction clusters the particles) grows them, runs the tuner
    again and steps on: the trajectory is the cell walk's bit for bit, and the
    step count ends at the target."""
    w = configs.config2()
    steps = 4000
    res = {}
    for mode in ("cells", "auto"):
        with Engine(w.system, precision="f32c", seed=3, neighbour_mode=mode) as e:
            e.set_particles(w.xyz, w.types)
            e.autotune()
            cap0 = e.metrics()["list_capacity"]
            e.step(steps)
            m = e.metrics()
            res[mode] = (e.get_particles()[0], cap0, m)
    xc, _, mc = res["cells"]
    xa, cap0, ma = res["auto"]
    assert mc["step"] == steps and ma["step"] == steps
    if ma["neighbour_mode"] == "list":
        assert ma["list_capacity"] > cap0, (cap0, ma["list_capacity"])
    assert np.array_equal(xc, xa)
