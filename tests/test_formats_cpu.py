"""Model and field formats of the reference, without a GPU.

* .fld (save_as_binary_fld / load, .jarvis_0_meta/.jarvis_2_field/
  jarvis_1_host_field_meat.hpp:41-64,81-89): the reference Frame's 72 bytes,
  then the data.  Files written by libjv (jv_fld_write) read back in Python
  and the other way round, bit for bit; the Frame's derived members and its
  type follow Frame(n, d, l) and set_frame_type (jarvis_0_frame_meat.hpp).
* raw models (host_single_field::read_raw, jarvis_1_host_field_meat.hpp:65-79):
  jv_raw_read takes exactly n floats and refuses a file of another size; a
  project with the raw-model argfile keys reads back through
  jv_read_argfile, and a raw-model key set without its frame is refused.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import pkg

jv = pkg()
project = pkg("project")


@pytest.mark.parametrize("shape,d,l,typ", [
    ((5, 1, 1), (0, 0, 0), (0, 0, 0), 1),         # vec
    ((4, 3, 1), (0, 0, 0), (0, 0, 0), 2),         # mat
    ((4, 3, 2), (0, 0, 0), (0, 0, 0), 3),         # cube
    ((6, 1, 1), (2.5, 0, 0), (1, 0, 0), 10),      # line
    ((1, 5, 4), (0, 3, 3), (0, -2, 7), 20),       # mesh
    ((7, 5, 3), (10, 10, 20), (-50, -50, 0), 30), # grid
])
def test_frame_matches_the_reference_construction(shape, d, l, typ):
    nx, ny, nz = shape
    f = jv.make_frame(nx, ny, nz, d, l)
    p = project.frame(nx, ny, nz, d, l)
    assert C.sizeof(jv.Frame) == 72 == project.FRAME.size
    assert f.type == p["type"] == typ
    assert (f.n_elem, f.n_rows, f.n_elem_slice, f.n_cols, f.n_slices) == (nx * ny * nz, nx, nx * ny, ny, nz)
    for a, nm in enumerate(("rows", "cols", "slices")):
        assert getattr(f, "r_" + nm) == p["r"][a] == np.float32(l[a] + (shape[a] - 1) * np.float32(d[a]))
        assert getattr(f, "l_" + nm) == p["l"][a]


def test_fld_round_trip_both_ways(tmp_path):
    rng = np.random.default_rng(4)
    a = rng.standard_normal((6, 5, 7)).astype(np.float32)
    d, l = (10.0, 10.0, 5.0), (0.0, -20.0, 3.5)
    # libjv writes, Python reads
    f = jv.make_frame(7, 5, 6, d, l)
    p1 = jv.fld_write(str(tmp_path / "c_written"), f, a)
    fr, b = project.read_fld(p1)
    assert np.array_equal(a, b) and fr["type"] == 30 and fr["n_rows"] == 7 and fr["n_slices"] == 6
    # Python writes, libjv reads: the same bytes
    p2 = project.write_fld(str(tmp_path / "py_written"), a, d, l)
    assert open(p1, "rb").read() == open(p2, "rb").read()
    f2, c = jv.fld_read(p2)
    assert np.array_equal(a, c) and bytes(f2) == bytes(f)


def test_fld_read_refuses_bad_input(tmp_path):
    L = jv.lib()
    f = jv.Frame()
    assert L.jv_fld_read(str(tmp_path / "x.raw").encode(), C.byref(f), None, 0) == jv.JV_EINVAL
    assert L.jv_fld_read(str(tmp_path / "missing.fld").encode(), C.byref(f), None, 0) == jv.JV_EIO
    p = project.write_fld(str(tmp_path / "small"), np.ones((2, 2, 2), np.float32))
    buf = np.empty(4, np.float32)
    assert L.jv_fld_read(p.encode(), C.byref(f), buf.ctypes.data_as(C.POINTER(C.c_float)), 4) == jv.JV_EINVAL
    with open(str(tmp_path / "trunc.fld"), "wb") as fh:
        fh.write(open(p, "rb").read()[:80])
    big = np.empty(8, np.float32)
    assert L.jv_fld_read(str(tmp_path / "trunc.fld").encode(), C.byref(f), big.ctypes.data_as(C.POINTER(C.c_float)),
                         8) == jv.JV_EIO


def test_raw_read_takes_exactly_n_values(tmp_path):
    L = jv.lib()
    a = np.arange(24, dtype=np.float32)
    path = str(tmp_path / "m.raw")
    a.tofile(path)
    out = np.zeros(24, np.float32)
    fp = out.ctypes.data_as(C.POINTER(C.c_float))
    assert L.jv_raw_read(path.encode(), 24, fp) == jv.JV_OK and np.array_equal(out, a)
    assert L.jv_raw_read(path.encode(), 23, fp) == jv.JV_EIO
    assert b"bytes" in L.jv_last_error()


def test_raw_model_project_keys(tmp_path, synth):
    s = synth.small_case(n=(12, 10, 9), pml=5, nt=20, seed=2)
    d = str(tmp_path / "proj") + "/"
    project.write_project(d, s, raw_model=True, save_fld=True)
    a = jv.read_argfile(d)
    assert a["vp_path"] == d + "vp.raw" and a["rho_path"] == d + "rho.raw"
    assert (a["n_rows"], a["n_cols"], a["n_slices"]) == (12, 10, 9)
    assert a["d_rows"] == pytest.approx(s.dx) and a["save_fld"] == 1
    vp = np.fromfile(a["vp_path"], dtype=np.float32).reshape(9, 10, 12)
    assert np.array_equal(vp, s.vp)
    # a raw model without its frame is refused
    txt = open(d + "argfile.json").read().replace('"n_rows": 12', '"n_rows": 0')
    open(d + "argfile.json", "w").write(txt)
    with pytest.raises(jv.JvError) as e:
        jv.read_argfile(d)
    assert e.value.code == jv.JV_EIO and "n_rows" in str(e.value)
