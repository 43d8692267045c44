"""The drop-in boundary: the XML input reader and the JNI entry point
Java_readdy_impl_sim_top_TopGPU_cCreateSimulation driven by a fake JNIEnv."""
import ctypes as C
import os

import numpy as np
import pytest

from readdygpu_b200 import _abi as A
from tests.fake_jni import FakeJVM, write_inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JNI_LIB = os.path.join(ROOT, "readdygpu_b200", "libCReaDDyGPU.so")


def jni_lib():
    import readdygpu_b200  # noqa: F401  (engine library first)
    return C.CDLL(JNI_LIB)


class RunParams(C.Structure):
    _fields_ = [("n_frames", C.c_int64), ("steps_per_frame", C.c_int64), ("dt_frame", C.c_double),
                ("device", C.c_int32), ("testmode", C.c_int32), ("n_unsupported", C.c_int32),
                ("reserved", C.c_int32)]


def inputs_lib():
    L = jni_lib()
    V, I64P, I32P = C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int32)
    L.rdgpu_inputs_read.restype = C.c_int
    L.rdgpu_inputs_read.argtypes = [C.c_char_p] * 4 + [C.c_double, C.POINTER(C.c_void_p)]
    L.rdgpu_inputs_read_groups.restype = C.c_int
    L.rdgpu_inputs_read_groups.argtypes = [V, C.c_char_p, C.c_char_p]
    L.rdgpu_inputs_bond_counts.restype = C.c_int
    L.rdgpu_inputs_bond_counts.argtypes = [V, I64P, I32P, I32P]
    L.rdgpu_inputs_bonds.restype = C.c_int
    L.rdgpu_inputs_bonds.argtypes = [V, I32P, I32P, C.POINTER(A.PairPot)]
    L.rdgpu_inputs_error.restype = C.c_char_p
    L.rdgpu_inputs_error.argtypes = [V]
    L.rdgpu_inputs_free.restype = None
    L.rdgpu_inputs_free.argtypes = [V]
    return L


def read_inputs(paths, max_cutoff=10.0):
    L = jni_lib()
    L.rdgpu_inputs_read.restype = C.c_int
    L.rdgpu_inputs_read.argtypes = [C.c_char_p] * 4 + [C.c_double, C.POINTER(C.c_void_p)]
    L.rdgpu_inputs_error.restype = C.c_char_p
    L.rdgpu_inputs_error.argtypes = [C.c_void_p]
    L.rdgpu_inputs_count.restype = C.c_int64
    L.rdgpu_inputs_count.argtypes = [C.c_void_p]
    h = C.c_void_p()
    rc = L.rdgpu_inputs_read(paths["param_particles"].encode(), paths["tplgy_potentials"].encode(),
                             paths["param_global"].encode(), paths["tplgy_coordinates"].encode(), max_cutoff,
                             C.byref(h))
    if rc:
        return rc, L.rdgpu_inputs_error(None).decode(), None, None, None
    d = A.SystemDesc()
    run = RunParams()
    L.rdgpu_inputs_desc(h, C.byref(d), C.byref(run))
    n = L.rdgpu_inputs_count(h)
    xyz = np.empty((n, 3))
    types = np.empty(n, np.int32)
    ids = np.empty(n, np.int32)
    L.rdgpu_inputs_particles(h, xyz.ctypes.data_as(C.c_void_p), types.ctypes.data_as(C.c_void_p),
                             ids.ctypes.data_as(C.c_void_p))
    L.rdgpu_inputs_free(h)
    return 0, d, run, (xyz, types, ids), None


def test_jni_symbol_exported():
    lib = jni_lib()
    assert hasattr(lib, "Java_readdy_impl_sim_top_TopGPU_cCreateSimulation")
    for n in ("rdgpu_inputs_read", "rdgpu_inputs_desc", "rdgpu_inputs_count", "rdgpu_inputs_particles",
              "rdgpu_inputs_error", "rdgpu_inputs_free"):
        assert hasattr(lib, n)


def test_input_files_parse(tmp_path):
    paths, xyz, types = write_inputs(tmp_path, n=50, frames=7)
    rc, d, run, parts, _ = read_inputs(paths)
    assert rc == 0
    M = A.MAX_TYPES
    assert d.n_types == 2
    assert d.D[0] == 1e6 and d.D[1] == 0.5e6
    assert d.p_radius[0] == 1.5 and d.p_radius[1] == 2.0
    # type B is 1.75 against A, A has its default 1.5 against B
    assert d.coll_radius[1 * M + 0] == 1.75 and d.coll_radius[0 * M + 1] == 1.5
    assert d.n_pair == 2 and d.n_ext == 1
    assert d.pair[0].kind == A.P2_HARMONIC and d.pair[0].subtype == A.SUB_REPULSIVE
    assert all(d.pair[0].pairs[i * M + j] for i in range(2) for j in range(2))
    assert d.pair[1].kind == A.P2_WEAK_PIECEWISE and d.pair[1].depth == 2 and d.pair[1].length == 1.3
    assert d.pair[1].pairs[0 * M + 1] and not d.pair[1].pairs[0]
    assert d.ext[0].kind == A.P1_CUBE and d.ext[0].consider_radius == 1 and d.ext[0].types[0] and d.ext[0].types[1]
    assert run.n_frames == 7 and run.steps_per_frame == 100 and d.dt == 1e-9
    assert abs(d.T - 293.15) < 1e-12 and d.kB == 0.0083144621
    assert list(d.lo) == [-20.0] * 3 and list(d.hi) == [20.0] * 3 and list(d.periodic) == [1, 1, 1]
    assert d.max_cutoff == 10.0
    x, t, ids = parts
    np.testing.assert_array_equal(x, xyz)
    np.testing.assert_array_equal(t, types)
    np.testing.assert_array_equal(ids, 1000 + np.arange(50))


def test_input_errors(tmp_path):
    paths, _, _ = write_inputs(tmp_path, n=5)
    bad = dict(paths)
    bad["param_global"] = str(tmp_path / "missing.xml")
    rc, msg, *_ = read_inputs(bad)
    assert rc == A.ERR_ARG and "cannot read" in msg
    open(tmp_path / "broken.xml", "w").write("<param_particles><particle></param_particles>")
    bad = dict(paths)
    bad["param_particles"] = str(tmp_path / "broken.xml")
    rc, msg, *_ = read_inputs(bad)
    assert rc == A.ERR_ARG and "mismatched" in msg


def test_input_refuses_cubic_weak_interaction(tmp_path):
    """The reference GPU runs WEAK_INTERACTION_HARMONIC (CudaSimulation.cu:1021-1031);
    this core does not implement it and refuses the input instead of skipping it."""
    paths, _, _ = write_inputs(tmp_path, n=5)
    for name in ("WEAK_INTERACTION_HARMONIC", "WEAK_INTERACTION"):
        txt = open(paths["tplgy_potentials"]).read()
        pot = (f'<pot name="cubic" type="{name}" forceConst="10" affectedParticleTypeIdPairs="[[0,1]]" '
               'affectedParticleIdPairs="" />\n</tplgy_potentials>')
        bad = dict(paths)
        bad["tplgy_potentials"] = str(tmp_path / f"pots_{name}.xml")
        open(bad["tplgy_potentials"], "w").write(txt.replace("</tplgy_potentials>", pot))
        rc, msg, *_ = read_inputs(bad)
        assert rc == A.ERR_ARG and name in msg and "not supported" in msg


def test_jni_without_device_reports_and_returns(tmp_path, capfd):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    paths, _, _ = write_inputs(tmp_path, n=20)
    frames = []
    jvm = FakeJVM(lambda f, a: frames.append(f) or True)
    jvm.run(jni_lib(), paths)
    out = capfd.readouterr().out
    assert "error during initialization" in out and "no CPU fallback" in out
    assert frames == []
    assert "UNEXPECTED" not in jvm.calls


@pytest.mark.gpu
def test_jni_protocol_frames_and_reactions(tmp_path, capfd):
    """Frame callbacks carry [N, (x,y,z,gpuIndex,readdyId) x N]; reactions in
    cReactions delete slots and append particles (ReaDDyGPU.cpp:264-463)."""
    n0 = 400
    paths, xyz, types = write_inputs(tmp_path, n=n0, frames=4)
    seen = {}

    def on_frame(frame, arr):
        n = int(arr[0])
        rec = arr[1:].reshape(n, 5)
        seen[frame] = rec
        return True

    def reactions(frame):
        if frame == 1:
            # delete gpu slots 3 and 10, turn slot 20 into a B, create one A
            return [4, 77, -1, 0, 0, 0, 3, 78, -1, 0, 0, 0, 10, 5000, 1, 1.0, 2.0, 3.0, 20,
                    5001, 0, -4.0, 5.0, 6.0, -1]
        return [0]

    jvm = FakeJVM(on_frame, reactions)
    jvm.run(jni_lib(), paths)
    out = capfd.readouterr().out
    assert "END" in out and "error" not in out.lower()
    assert "UNEXPECTED" not in jvm.calls
    assert sorted(seen) == [0, 1, 2, 3]
    r0, r1, r2 = seen[0], seen[1], seen[2]
    assert len(r0) == n0 and len(r1) == n0
    np.testing.assert_array_equal(r0[:, 3], np.arange(n0))
    np.testing.assert_array_equal(r0[:, 4], 1000 + np.arange(n0))
    # particles moved by diffusion, but stayed near their start (100 steps of ~0.045 nm)
    d = r0[:, :3] - xyz.astype(np.float32)
    assert 0 < np.abs(d).max() < 5.0
    # frame 2: 400 - 3 deleted + 2 created
    assert len(r2) == n0 - 1
    ids2 = r2[:, 4].astype(int).tolist()
    assert 1003 not in ids2 and 1010 not in ids2 and 1020 not in ids2
    assert ids2[-2:] == [5000, 5001]
    np.testing.assert_array_equal(r2[:, 3], np.arange(n0 - 1))
    assert np.abs(r2[-2, :3] - [1.0, 2.0, 3.0]).max() < 1.0


def test_input_groups_as_bonds(tmp_path):
    """param_groups / tplgy_groups become bonded pairs: one spring per dimer
    instance, gpu indices from the particle ids; unsupported group potentials
    are counted and skipped."""
    paths, _, _ = write_inputs(tmp_path, n=50, dimers=5)
    L = inputs_lib()
    h = C.c_void_p()
    assert L.rdgpu_inputs_read(paths["param_particles"].encode(), paths["tplgy_potentials"].encode(),
                               paths["param_global"].encode(), paths["tplgy_coordinates"].encode(), 10.0,
                               C.byref(h)) == 0
    assert L.rdgpu_inputs_read_groups(h, paths["param_groups"].encode(), paths["tplgy_groups"].encode()) == 0
    nb, npot, nu = C.c_int64(), C.c_int32(), C.c_int32()
    L.rdgpu_inputs_bond_counts(h, C.byref(nb), C.byref(npot), C.byref(nu))
    assert (nb.value, npot.value, nu.value) == (5, 1, 1)
    ij = (C.c_int32 * 10)()
    pot = (C.c_int32 * 5)()
    pots = (A.PairPot * 1)()
    L.rdgpu_inputs_bonds(h, ij, pot, pots)
    assert list(ij) == [0, 1, 2, 3, 4, 5, 6, 7, 8, 9] and list(pot) == [0] * 5
    assert pots[0].kind == A.P2_HARMONIC and pots[0].subtype == A.SUBTYPES["spring"] and pots[0].k == 20.0
    assert pots[0].r0 == -1.0
    # a group instance naming an unknown particle id is an error
    open(paths["tplgy_groups"], "w").write('<tplgy_groups><g id="0" type="0" internalAndParticleId="[[0,5];[1,6]]"/></tplgy_groups>')
    assert L.rdgpu_inputs_read_groups(h, paths["param_groups"].encode(), paths["tplgy_groups"].encode()) != 0
    assert b"unknown particle id" in L.rdgpu_inputs_error(h)
    L.rdgpu_inputs_free(h)


@pytest.mark.gpu
def test_jni_groups_hold_dimers_together(tmp_path, capfd):
    """Spring-bonded dimers from the group files stay at about their rest
    length (3 nm, sqrt(kT/k) = 0.35 nm) through the frames."""
    paths, _, _ = write_inputs(tmp_path, n=200, frames=5, dimers=20)
    seen = {}
    jvm = FakeJVM(lambda f, a: seen.__setitem__(f, a.copy()) or True)
    jvm.run(jni_lib(), paths)
    out = capfd.readouterr().out
    assert "END" in out and "error" not in out.lower()
    rec = seen[4][1:].reshape(-1, 5)
    d = np.linalg.norm(rec[0:40:2, :3] - rec[1:40:2, :3], axis=1)
    assert np.all(np.abs(d - 3.0) < 2.0), d


@pytest.mark.gpu
def test_jni_callback_false_stops(tmp_path, capfd):
    paths, _, _ = write_inputs(tmp_path, n=100, frames=5)
    seen = []
    jvm = FakeJVM(lambda f, a: seen.append(f) or f < 1)
    jvm.run(jni_lib(), paths)
    out = capfd.readouterr().out
    assert seen == [0, 1]
    assert "error in java" in out
