"""The jarvis-named C++ front end (include/jv/jarvis_compat.hpp) without a
GPU: drivers in the reference's shape compile and link against libjv.so,
and the argfile reader behind ArgList::mpi_read_arg_file reads the
reference's schema."""
import subprocess

import pytest

from conftest import build_compat_driver, pkg

jv = pkg()


@pytest.mark.parametrize("name", ["rtm_main", "forward_main"])
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
