"""Trajectory and RDF writers (include/readdy_b200_output.h) against the
formats of the reference's outputHandler (outputHandler.cpp:19-148), and the
XML trajectory as a restart file through the coordinate reader.  Host code
only: no GPU."""
import ctypes as C
import re

import numpy as np
import pytest

from .fake_jni import write_inputs
from .test_abi import declared
from .test_jni_shim import jni_lib, read_inputs

XML, PDB = 0, 1


def out_lib():
    L = jni_lib()
    V = C.c_void_p
    L.rdgpu_traj_open.restype = C.c_int
    L.rdgpu_traj_open.argtypes = [C.c_char_p, C.c_int32, C.POINTER(V)]
    L.rdgpu_traj_write.restype = C.c_int
    L.rdgpu_traj_write.argtypes = [V, C.c_int64, C.c_int64, V, V, V]
    L.rdgpu_traj_close.restype = C.c_int
    L.rdgpu_traj_close.argtypes = [V]
    L.rdgpu_write_rdf_csv.restype = C.c_int
    L.rdgpu_write_rdf_csv.argtypes = [C.c_char_p, C.c_int32, C.POINTER(C.c_char_p), C.c_int32, C.c_double, V]
    L.rdgpu_output_error.restype = C.c_char_p
    L.rdgpu_output_error.argtypes = []
    return L


def ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def write_traj(path, fmt, frames):
    L = out_lib()
    h = C.c_void_p()
    assert L.rdgpu_traj_open(str(path).encode(), fmt, C.byref(h)) == 0
    for step, xyz, types, ids in frames:
        xyz = np.ascontiguousarray(xyz, np.float64)
        types = np.ascontiguousarray(types, np.int32)
        ids = None if ids is None else np.ascontiguousarray(ids, np.int32)
        assert L.rdgpu_traj_write(h, step, len(types), ptr(xyz), ptr(types), ptr(ids)) == 0
    assert L.rdgpu_traj_close(h) == 0


def test_output_exports_every_declared_symbol():
    lib = jni_lib()
    names = declared("readdy_b200_output.h")
    assert len(names) == 5
    for n in names:
        assert hasattr(lib, n), n


def test_xml_trajectory_format(tmp_path):
    p = tmp_path / "traj.xml"
    xyz = np.array([[1.5, -2.25, 3.0], [0.1, 0.2, 0.3]])
    write_traj(p, XML, [(0, xyz, [0, 1], None), (100, xyz + 1, [0, 1], [7, 9])])
    lines = p.read_text().splitlines()
    assert lines[0] == "<traj>" and lines[-1] == "</traj>"
    assert lines[1] == '<tplgy_coords version="1.1" stepId="0">'
    assert lines[2] == '<p id="1" type="0" c="1.5,-2.25,3"/>'
    assert lines[3] == '<p id="2" type="1" c="0.10000000000000001,0.20000000000000001,0.29999999999999999"/>'
    assert lines[4] == "</tplgy_coords>"
    assert lines[5] == '<tplgy_coords version="1.1" stepId="100">'
    assert lines[6].startswith('<p id="7" type="0" c="2.5,')


def test_xml_trajectory_restarts_bit_for_bit(tmp_path):
    """The last frame of a trajectory, read back as tplgy_coordinates, gives
    the written state exactly (17 significant digits)."""
    paths, xyz0, types = write_inputs(tmp_path, n=60)
    rng = np.random.default_rng(3)
    x1 = rng.uniform(-20, 20, (60, 3))
    x2 = x1 + rng.normal(0, 1e-7, (60, 3))      # differences below the reference's 3 decimals
    ids = 1000 + np.arange(60)
    p = tmp_path / "traj.xml"
    write_traj(p, XML, [(0, x1, types, ids), (500, x2, types, ids)])
    paths = dict(paths, tplgy_coordinates=str(p))
    rc, d, run, parts, _ = read_inputs(paths)
    assert rc == 0
    x, t, i = parts
    np.testing.assert_array_equal(x, x2)
    np.testing.assert_array_equal(t, types)
    np.testing.assert_array_equal(i, ids)


def test_xml_trajectory_without_frames_is_an_error(tmp_path):
    paths, _, _ = write_inputs(tmp_path, n=10)
    p = tmp_path / "empty.xml"
    write_traj(p, XML, [])
    rc, msg, *_ = read_inputs(dict(paths, tplgy_coordinates=str(p)))
    assert rc != 0 and "traj" in msg


def test_pdb_trajectory_format(tmp_path):
    p = tmp_path / "traj.pdb"
    xyz = np.array([[1.0, 2.0, 3.0], [-10.5, 0.0, 123.4567]])
    write_traj(p, PDB, [(3, xyz, [0, 2], None)])
    lines = p.read_text().splitlines()
    assert lines[0] == "MODEL     3" and lines[-1] == "ENDMDL"
    assert lines[1] == "ATOM      1   0    0     1       1.000   2.000   3.000 15.00  0.00"
    assert lines[2] == "ATOM      2   2    2     1     -10.500   0.000 123.457 15.00  0.00"
    # PDB columns: x, y, z in 31-38, 39-46, 47-54 (1-based)
    assert float(lines[2][30:38]) == -10.5 and float(lines[2][46:54]) == 123.457


def test_rdf_csv_format(tmp_path):
    L = out_lib()
    S, nb, rmax = 2, 4, 2.0
    g = np.arange(S * S * nb, dtype=np.float64) * 0.5
    names = (C.c_char_p * S)(b"A", b"B")
    p = tmp_path / "rdf.csv"
    assert L.rdgpu_write_rdf_csv(str(p).encode(), S, names, nb, rmax, ptr(g)) == 0
    lines = p.read_text().splitlines()
    assert lines[0] == "d,\tRDF(A,A),\tRDF(A,B),\tRDF(B,A),\tRDF(B,B)"
    assert len(lines) == 1 + nb
    for k in range(nb):
        cols = [float(c) for c in lines[k + 1].split(",")]
        assert cols[0] == k * rmax / nb
        assert cols[1:] == [g[(a * S + b) * nb + k] for a in range(S) for b in range(S)]
    assert re.fullmatch(r" 0\.50000,    0\.500,    2\.500,    4\.500,    6\.500", lines[2])


def test_writer_errors(tmp_path):
    L = out_lib()
    h = C.c_void_p()
    assert L.rdgpu_traj_open(str(tmp_path / "x.xml").encode(), 7, C.byref(h)) < 0
    assert b"format" in L.rdgpu_output_error()
    assert L.rdgpu_traj_open(str(tmp_path / "no_dir" / "x.xml").encode(), XML, C.byref(h)) < 0
    assert b"cannot open" in L.rdgpu_output_error()
    names = (C.c_char_p * 1)(b"A")
    g = np.zeros(4)
    assert L.rdgpu_write_rdf_csv(str(tmp_path / "r.csv").encode(), 1, names, 0, 1.0, ptr(g)) < 0
    assert L.rdgpu_write_rdf_csv(str(tmp_path / "r.csv").encode(), 1, names, 4, -1.0, ptr(g)) < 0
    assert L.rdgpu_traj_open(str(tmp_path / "x.xml").encode(), XML, C.byref(h)) == 0
    assert L.rdgpu_traj_write(h, 0, 3, None, None, None) < 0
    assert L.rdgpu_traj_close(h) == 0
