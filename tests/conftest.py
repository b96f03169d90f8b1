"""Shared fixtures: import paths for the package (its directory name has
hyphens, so it is imported with importlib) and the oracle, and the gpu
marker.  `-m "not gpu"` runs on any machine; `-m gpu` needs a CUDA device
and the built libjv.so."""
import importlib
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)

PKG = "domain-decomposition-release_b200"


def pkg(mod: str = ""):
    return importlib.import_module(PKG + ("." + mod if mod else ""))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built libjv.so")


@pytest.fixture(scope="session")
def synth():
    return pkg("synth")


@pytest.fixture(scope="session")
def project():
    return pkg("project")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib("f64")
    O.lib("f32")
    return O


def rel_l2(a, b):
    import numpy as np
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


def build_compat_driver(name: str, out_dir: str) -> str:
    """Compiles tests/compat/<name>.cpp (a driver written against the jarvis
    class names) against include/jv/jarvis_compat.hpp and libjv.so."""
    import subprocess
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    libdir = os.path.join(ROOT, PKG)
    exe = os.path.join(out_dir, name)
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(cuda, "include"), os.path.join(ROOT, "tests", "compat", name + ".cpp"),
           "-L", libdir, "-ljv", "-L", os.path.join(cuda, "lib64"), "-lcudart", f"-Wl,-rpath,{libdir}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe
