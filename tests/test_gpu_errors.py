"""A step that blows up: the error names the failing step, and the handle
keeps that step's input (later steps of the same CUDA graph did nothing), in
both neighbour modes and both precisions, inside and outside a graph."""
import numpy as np
import pytest

from readdygpu_b200 import _abi as A, RdgpuError
from readdygpu_b200.system import PairPotential

from .test_gpu_parity import Engine, cfg1

pytestmark = pytest.mark.gpu

# a stiff spring at rest: step 0 moves the pair by noise only, then the
# spring (k = 1e9) throws both particles many box lengths away in step 1
STIFF = [PairPotential(A.P2_HARMONIC, [], 1e9, "spring", r0=3.0)]


def blowup_system():
    sys_, xyz, types = cfg1(200)
    xyz = xyz.copy()
    xyz[1] = xyz[0] + [3.0, 0.0, 0.0]
    xyz[1] = np.mod(xyz[1], 50.0)
    return sys_, xyz, types


@pytest.mark.parametrize("prec", ["f64", "f32c"])
@pytest.mark.parametrize("mode", ["cells", "list"])
@pytest.mark.parametrize("nsteps", [5, 250])
def test_blowup_reports_step_and_keeps_its_input(prec, mode, nsteps):
    sys_, xyz, types = blowup_system()
    with Engine(sys_, precision=prec, seed=3, neighbour_mode=mode, skin=0.8) as ref:
        ref.set_particles(xyz, types)
        ref.set_bonds([[0, 1]], [0], STIFF)
        ref.step(1)
        x1, _ = ref.get_particles()
    with Engine(sys_, precision=prec, seed=3, neighbour_mode=mode, skin=0.8) as e:
        e.set_particles(xyz, types)
        e.set_bonds([[0, 1]], [0], STIFF)
        with pytest.raises(RdgpuError) as ex:
            e.step(nsteps)
        assert ex.value.code in (A.ERR_JUMP, A.ERR_NONFINITE)
        assert "at step 1" in str(ex.value)
        assert e.metrics()["step"] == 1
        x, _ = e.get_particles()
        np.testing.assert_array_equal(x, x1)
        # the handle stays usable: a fresh upload steps normally
        e.set_particles(xyz, types)
        e.step(20)
        assert np.isfinite(e.get_particles()[0]).all()
