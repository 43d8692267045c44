"""Reaction edits on the device (rdgpu_apply_edits) against the reference's
host-side semantics (ReaDDyGPU.cpp:303-461): delete by gpu index, append new
particles, survivors keep their order, appended ones follow, indices are
renumbered.  Survivors keep their stored state bit for bit."""
import numpy as np
import pytest

from readdygpu_b200 import _abi as A

from .test_gpu_parity import Engine, cfg1, oracle_state

pytestmark = pytest.mark.gpu


def edits(deletes=(), appends=()):
    rows = []
    for i, g in enumerate(deletes):
        rows.append([100 + i, -1, 0, 0, 0, g])
    for i, (t, x, y, z) in enumerate(appends):
        rows.append([500 + i, t, x, y, z, -1])
    return np.array(rows, dtype=np.float32).reshape(-1, 6)


def expected(x1, t1, deletes, appends):
    keep = np.ones(len(t1), bool)
    keep[list(deletes)] = False
    xa = np.array([[x, y, z] for (_, x, y, z) in appends], dtype=np.float32).astype(np.float64).reshape(-1, 3)
    ta = np.array([t for (t, _, _, _) in appends], dtype=np.int32)
    return np.concatenate([x1[keep], xa]), np.concatenate([t1[keep], ta])


DEL = (0, 7, 123, 999)
APP = ((1, 10.5, 20.25, 30.0), (0, 0.5, 49.5, 25.0), (1, 25.0, 25.0, 25.0))


@pytest.mark.parametrize("prec", ["f64", "f32c"])
@pytest.mark.parametrize("mode", ["cells", "list"])
def test_edits_delete_append_renumber(oracle, prec, mode):
    sys_, xyz, types = cfg1(1000)
    with Engine(sys_, precision=prec, seed=4, neighbour_mode=mode, skin=0.8) as e:
        e.set_particles(xyz, types)
        e.step(60)
        x1, t1 = e.get_particles()
        e.apply_edits(edits(DEL, APP))
        assert e.n == 1000 - len(DEL) + len(APP)
        x2, t2 = e.get_particles()
        cnt, h = e.neighbor_digest()
        F, _ = e.forces()
        e.step(40)      # the edited state steps on
        x3, _ = e.get_particles()
        m = e.metrics()
    xe, te = expected(x1, t1, DEL, APP)
    np.testing.assert_array_equal(t2, te)
    nk = 1000 - len(DEL)
    # survivors: their stored state is moved, not recomputed
    np.testing.assert_array_equal(x2[:nk], xe[:nk])
    tol = 0.0 if prec == "f64" else 4e-6
    assert np.abs(x2[nk:] - xe[nk:]).max() <= tol
    assert m["step"] == 100
    d = x3 - x2
    d -= 50.0 * np.round(d / 50.0)   # periodic 50 nm cube
    assert np.isfinite(x3).all() and np.abs(d).max() < 2.0
    if prec == "f64":
        d, stored, _ = oracle_state(oracle, sys_, x2, "f64")
        ocnt, oh = oracle.neighbor_digest(d, stored, t2, f32=False)
        assert np.array_equal(cnt, ocnt) and np.array_equal(h, oh)
        Fo, _ = oracle.forces_f64(d, stored, t2)
        assert np.linalg.norm(F - Fo) <= 1e-10 * np.linalg.norm(Fo)


def test_edits_list_and_cells_trajectories_identical():
    """FP32C: the same edits in both neighbour modes, then steps: bit-identical."""
    sys_, xyz, types = cfg1(2000)
    out = []
    for mode in ("cells", "list"):
        with Engine(sys_, precision="f32c", seed=8, neighbour_mode=mode, skin=0.6) as e:
            e.set_particles(xyz, types)
            e.step(50)
            e.apply_edits(edits((5, 6, 1999), ((0, 1.0, 1.0, 1.0),)))
            e.step(120)
            e.apply_edits(edits((0,), ((1, 40.0, 40.0, 40.0), (1, 41.0, 40.0, 40.0))))
            e.step(30)
            out.append(e.get_particles())
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])


def test_edits_growth_keeps_state():
    """Appending beyond the buffers' headroom grows them and keeps the state."""
    sys_, xyz, types = cfg1(400)
    rng = np.random.default_rng(3)
    app = [(int(rng.integers(0, 2)), *rng.uniform(0, 50, 3)) for _ in range(300)]
    with Engine(sys_, precision="f32c", seed=2) as e:
        e.set_particles(xyz, types)
        e.step(20)
        x1, t1 = e.get_particles()
        m1 = e.metrics()
        e.apply_edits(edits((), app))
        assert e.n == 700
        x2, t2 = e.get_particles()
        m2 = e.metrics()
        e.step(20)
    np.testing.assert_array_equal(x2[:400], x1)
    np.testing.assert_array_equal(t2[:400], t1)
    # appended particles start their MSD at their position: per type
    # msd_after = msd_before * n_before / n_after
    for t in range(2):
        nb = np.sum(t1 == t)
        na = np.sum(t2 == t)
        assert abs(m2["msd"][t] - m1["msd"][t] * nb / na) <= 1e-9 * max(1.0, m1["msd"][t])


def test_edits_errors_leave_state():
    sys_, xyz, types = cfg1(300)
    with Engine(sys_, precision="f64") as e:
        e.set_particles(xyz, types)
        x1, _ = e.get_particles()
        for bad in (edits((300,)), edits((5, 5)), edits((), ((7, 1.0, 1.0, 1.0),)),
                    np.array([[0, 0.5, 0, 0, 0, -1]], np.float32)):
            with pytest.raises(RuntimeError):
                e.apply_edits(bad)
            assert e.n == 300
            np.testing.assert_array_equal(e.get_particles()[0], x1)
        e.apply_edits(np.zeros((0, 6), np.float32))
        np.testing.assert_array_equal(e.get_particles()[0], x1)


def test_edits_need_single_system():
    from readdygpu_b200 import configs
    w = configs.config4(n_systems=3, nmin=100, nmax=200)
    with Engine(w.system, precision="f32c", boxes=w.boxes) as e:
        e.set_particles(w.xyz, w.types, offsets=w.offsets)
        with pytest.raises(RuntimeError):
            e.apply_edits(edits((0,)))
