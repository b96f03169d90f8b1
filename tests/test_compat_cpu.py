"""The jarvis-named C++ front end (include/jv/jarvis_compat.hpp) without a
GPU: drivers in the reference's shape compile and link against libjv.so,
and the argfile reader behind ArgList::mpi_read_arg_file reads the
reference's schema."""
import subprocess

import pytest

from conftest import build_compat_driver, pkg

jv = pkg()


@pytest.mark.parametrize("name", ["rtm_main", "forward_main", "rtm_modules_main", "field_main"])
def test_driver_builds(tmp_path, name):
    build_compat_driver(name, str(tmp_path))


def test_driver_usage_without_device(tmp_path):
    exe = build_compat_driver("rtm_main", str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stdout


def test_read_argfile_prefixes_paths(tmp_path, project, synth):
    s = synth.small_case(n=(10, 10, 10), pml=4, nt=10)
    d = str(tmp_path / "p") + "/"
    project.write_project(d, s)
    a = jv.read_argfile(d)
    assert a["model_path"].startswith(d) and a["shot_path"].startswith(d) and a["output_path"].startswith(d)
    assert a["pml_num"] == 4 and a["x_divide_num"] == 1 and a["slots_per_node"] >= 1
    assert abs(a["dt"] - s.dt) < 1e-9 and abs(a["fm"] - s.fm) < 1e-6


def test_read_argfile_missing(tmp_path):
    with pytest.raises(jv.JvError) as e:
        jv.read_argfile(str(tmp_path) + "/")
    assert e.value.code == jv.JV_EIO


def test_frame_and_field_in_the_reference_formats(tmp_path, project):
    """Field::read_raw onto a grid Frame, save as .fld / .raw / ascii_xyz,
    Field::load of the .fld: the same frame and values; the files are the
    reference's formats (the .fld header is the Frame's 72 bytes)."""
    import numpy as np

    exe = build_compat_driver("field_main", str(tmp_path))
    d = str(tmp_path) + "/"
    a = np.arange(24, dtype=np.float32).reshape(2, 3, 4) * 0.5
    a.tofile(d + "in.raw")
    r = subprocess.run([exe, d], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    first = r.stdout.split("\n")[0].split()
    assert first[1] == "1" and first[3] == "30" and first[9] == "0", r.stdout
    assert [float(v) for v in first[5:8]] == [10.0, 20.0, 7.5]  # r = l + (n - 1) d
    assert first[11:] == ["2", "2", "1", "20"]  # Frame::sparse(2)
    want = a.copy()
    want[1, 2, 1] += 100.0
    fr, b = project.read_fld(d + "out.fld")
    assert np.array_equal(b, want) and fr["l"][0] == -20.0 and fr["d"][2] == 5.0
    suf = project.size_info(4, 3, 2, -20.0, 0.0, 2.5)
    assert r.stdout.split("\n")[1] == suf
    assert np.array_equal(np.fromfile(d + "out" + suf + ".raw", np.float32).reshape(2, 3, 4), want)
    rows = open(d + "out_xyz.txt").read().splitlines()
    assert len(rows) == 24 and rows[0].startswith("-20.000,  0.000,  2.500,")
