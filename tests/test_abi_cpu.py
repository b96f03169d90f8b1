"""The C ABI without a GPU: the library loads, exports every function
include/jv/jv.h declares, and rejects bad problems with status codes
before touching a device.  Project files round-trip in the reference's
formats."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT, pkg

jv = pkg()


def header_functions():
    txt = open(os.path.join(ROOT, "include", "jv", "jv.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(jv_[a-z_]+)\s*\(", txt)))


def test_library_exports_every_declared_function():
    L = jv.lib()
    names = header_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", jv.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (jv_\w+)", out))
    assert set(names) <= exported
    assert set(jv.EXPORTS) == set(names)


def test_build_info():
    assert b"sm_100a" in jv.lib().jv_build_info()


def _create(**kw):
    nx, ny, nz = kw.pop("n", (12, 12, 12))
    pml = kw.pop("pml", 5)
    a = np.full(nx * ny * nz, 2000.0, np.float32)
    args = dict(dt=1e-3, fm=20.0, nt=10)
    args.update(kw)
    return jv.Context.create(nx, ny, nz, pml, 10.0, 10.0, 10.0, a, a / 1.7, a, args["dt"], args["fm"], args["nt"],
                             **{k: v for k, v in args.items() if k not in ("dt", "fm", "nt")})


@pytest.mark.parametrize("kw,msg", [
    (dict(n=(7, 12, 12)), "at least 8"),
    (dict(pml=3), "pml_num must be >= 4"),
    (dict(dt=0.0), "dt and fm"),
    (dict(nt=0), "nt must be"),
    (dict(rec_width=5), "rec_width"),
    (dict(pml=4, rec_width=4, precision=7), "FP32"),
    (dict(min_blocks=5), "min_blocks"),
    (dict(pml_min_blocks=2), "min_blocks"),
    (dict(tile_gx=200, tile_gy=2), "tile_gx"),
    (dict(planes_per_thread=3), "planes_per_thread"),
    (dict(kernel_variant=5), "kernel_variant"),
])
def test_invalid_problems_rejected_without_device(kw, msg):
    with pytest.raises(jv.JvError) as e:
        _create(**kw)
    assert e.value.code in (jv.JV_EINVAL, jv.JV_ENOTSUP)
    assert msg in str(e.value)


def test_open_missing_project(tmp_path):
    with pytest.raises(jv.JvError) as e:
        jv.Context.open(str(tmp_path) + "/")
    assert e.value.code == jv.JV_EIO


def test_open_rejects_domain_split(tmp_path, project, synth):
    s = synth.small_case(n=(10, 10, 10), pml=4, nt=10)
    d = str(tmp_path / "p")
    project.write_project(d, s)
    txt = open(d + "/argfile.json").read().replace('"x_divide_num": 1', '"x_divide_num": 2')
    open(d + "/argfile.json", "w").write(txt)
    with pytest.raises(jv.JvError) as e:
        jv.Context.open(d + "/")
    assert e.value.code == jv.JV_EINVAL and "divide_num" in str(e.value)


def test_reference_example_argfile_parses(tmp_path, project):
    """The reference's own example argfile (JSON with // comments)."""
    text = """{
    "model_path": "cube100.gms",
    "shot_path": "shot.txt",
    "rece_path": "rece.txt",
    "output_path": "out/",
    //
    "is_output": false,
    //
    "pml_num": 10,
    "fm": 100,
    "dt": 0.0001,
    "T": 0.16,
    "t_snap": -1,
    //*mpi parameter
    //Grid Dividec
    "x_divide_num": 2,
    "y_divide_num": 2,
    "z_divide_num": 1,
    "slots_per_node": 4
}"""
    d = tmp_path / "ex"
    d.mkdir()
    (d / "argfile.json").write_text(text)
    a = project.read_argfile(str(d))
    assert a["model_path"] == str(d) + "/cube100.gms"
    assert a["pml_num"] == 10 and a["x_divide_num"] == 2 and a["slots_per_node"] == 4
    assert abs(a["T"] - 0.16) < 1e-7 and abs(a["dt"] - 1e-4) < 1e-9 and a["fm"] == 100
    assert a["rec_width"] == 1 and a["is_output"] is False


def test_gms_roundtrip(tmp_path, project, synth):
    s = synth.small_case(n=(11, 9, 7), pml=4, nt=5)
    p = str(tmp_path / "m.gms")
    project.write_gms(p, {"vp": s.vp, "vs": s.vs, "rho": s.rho}, d=(s.dx, s.dy, s.dz))
    m, g = project.read_gms(p)
    assert (g["nx"], g["ny"], g["nz"]) == (11, 9, 7) and g["dx"] == s.dx
    assert np.array_equal(m["vp"], s.vp) and np.array_equal(m["vs"], s.vs) and np.array_equal(m["rho"], s.rho)
    # z fastest, then x, then y on disk (jarvis_device_gms_meat.hpp:41-52)
    raw = np.fromfile(p, np.uint8)
    first = np.frombuffer(raw[240 + 64:240 + 64 + 8].tobytes(), np.float32)
    assert first[0] == s.vp[0, 0, 0] and first[1] == s.vp[1, 0, 0]


def test_traces_format(tmp_path, project):
    tr = np.array([[0.0, 1.5e-3, -2.25e-7], [3.0, -4.0, 5.0e10]], np.float32)
    p = project.write_traces(str(tmp_path / "vx_seis_0_0"), tr)
    line = open(p).readline()
    assert line == "0.000000e+00\t1.500000e-03\t-2.250000e-07\t\n"
    np.testing.assert_allclose(project.read_traces(p), tr, rtol=1e-6)


def test_size_info_matches_reference_naming(project):
    assert project.size_info(30, 26, 22) == "_30_26_22_0.000000_0.000000_0.000000"


def test_stream_probe_rejects_bad_arguments_without_device():
    jv = pkg()
    L = jv.lib()
    g = C.c_double()
    for nr, nw, n, reps in ((3, 3, 1024, 1), (1, 1, 1022, 1), (1, 1, 0, 1), (25, 11, 1024, 0)):
        assert L.jv_stream_probe(0, nr, nw, n, reps, C.byref(g)) == jv.JV_EINVAL
    assert L.jv_stream_probe(0, 1, 1, 1024, 1, None) == jv.JV_EINVAL
    assert b"(25,11)" in L.jv_last_error() or b"bad argument" in L.jv_last_error()


def test_python_structs_match_the_header(tmp_path):
    """Every ctypes mirror of a jv.h struct has the C layout: the size and
    each field's offset, from a C program compiled against the header."""
    jv = pkg()
    mirrors = {"jv_grid": jv.Grid, "jv_options": jv.Options, "jv_job": jv.Job, "jv_request": jv.Request,
               "jv_server_stats": jv.ServerStats, "jv_argfile": jv.ArgFileC, "jv_frame": jv.Frame,
               "jv_info": jv.Info}
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "jv/jv.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'    printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'    printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = {}
    for ln in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.splitlines():
        cname, key, val = ln.split()
        got[(cname, key)] = int(val)
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)
