"""ctypes wrapper around the CPU oracle (liboracle_f64.so / liboracle_f32.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by the CPU-baseline legs of ``bench.py``.  The product
(libjv.so and its Python mirror) never imports this module.

The oracle restates the reference's elastic FDTD modelling and VOWR RTM
(see jv_oracle.h for the file:line of every routine it follows).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def build() -> None:
    """Compile both oracle variants with the Makefile next to this file."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class _Problem(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("pml", C.c_int),
        ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float),
        ("dt", C.c_float), ("fm", C.c_float), ("T", C.c_float),
        ("rec_width", C.c_int),
        ("n_shot", C.c_int), ("shot_xyz", C.POINTER(C.c_float)),
        ("n_recv", C.c_int), ("recv_xyz", C.POINTER(C.c_float)),
        ("nthreads", C.c_int),
    ]


_LIBS: dict[str, C.CDLL] = {}


def lib(precision: str = "f64") -> C.CDLL:
    if precision not in ("f64", "f32"):
        raise ValueError(precision)
    if precision in _LIBS:
        return _LIBS[precision]
    path = os.path.join(HERE, f"liboracle_{precision}.so")
    if not os.path.exists(path):
        build()
    L = C.CDLL(path)
    dp = C.POINTER(C.c_double)
    fp = C.POINTER(C.c_float)
    P = C.POINTER(_Problem)
    L.jvo_ntime.argtypes = [C.c_float, C.c_float]
    L.jvo_ntime.restype = C.c_int
    L.jvo_diff_coeff.argtypes = [C.c_int, dp]
    L.jvo_ricker.argtypes = [C.c_int, C.c_float, C.c_float, fp]
    L.jvo_gap_num.argtypes = [C.c_float, C.c_float, C.c_float]
    L.jvo_gap_num.restype = C.c_int
    L.jvo_cpml_ab.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float, dp]
    L.jvo_cpml_ab.restype = C.c_int
    L.jvo_select_inside.argtypes = [P, fp, C.c_int, C.POINTER(C.c_int)]
    L.jvo_select_inside.restype = C.c_int
    L.jvo_forward.argtypes = [P, fp, fp, fp, C.c_int, dp, dp, dp]
    L.jvo_forward.restype = C.c_int
    L.jvo_rtm_shot.argtypes = [P, fp, fp, fp, C.c_int, dp, dp, dp, dp, dp, dp, dp, dp, dp]
    L.jvo_rtm_shot.restype = C.c_int
    L.jvo_finalize_image.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, dp, dp, dp, dp, dp]
    L.jvo_rtm_sample.argtypes = [P, fp, fp, fp, C.c_int, C.c_int]
    L.jvo_rtm_sample.restype = C.c_double
    L.jvo_set_store16.argtypes = [C.c_int]
    L.jvo_set_store16.restype = None
    _LIBS[precision] = L
    return L


def _f(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _d(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class Problem:
    """One modelling/RTM problem on gridphy (nx, ny, nz) + pml per face.

    shots / recvs are (n, 3) float32 arrays of positions in metres.
    vp, vs, rho are float32 arrays of shape (nz, ny, nx) (x fastest).
    """
    nx: int
    ny: int
    nz: int
    pml: int
    dx: float
    dy: float
    dz: float
    dt: float
    fm: float
    T: float
    rec_width: int
    shots: np.ndarray
    recvs: np.ndarray
    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    nthreads: int = 0
    _keep: list = field(default_factory=list, repr=False)

    def _c(self) -> _Problem:
        sh = np.ascontiguousarray(self.shots, dtype=np.float32).reshape(-1, 3)
        rc = np.ascontiguousarray(self.recvs, dtype=np.float32).reshape(-1, 3)
        self._keep = [sh, rc]
        return _Problem(self.nx, self.ny, self.nz, self.pml, self.dx, self.dy, self.dz, self.dt, self.fm,
                        self.T, self.rec_width, sh.shape[0], _f(sh), rc.shape[0], _f(rc), self.nthreads)

    def _model(self):
        m = [np.ascontiguousarray(a, dtype=np.float32) for a in (self.vp, self.vs, self.rho)]
        for a in m:
            if a.size != self.nx * self.ny * self.nz:
                raise ValueError("model array size does not match the grid")
        return m


def ntime(T: float, dt: float, precision: str = "f64") -> int:
    return lib(precision).jvo_ntime(T, dt)


def diff_coeff(order: int) -> np.ndarray:
    c = np.zeros(order, np.float64)
    lib().jvo_diff_coeff(order, _d(c))
    return c


def ricker(nt: int, fm: float, dt: float) -> np.ndarray:
    w = np.zeros(nt, np.float32)
    lib().jvo_ricker(nt, fm, dt, _f(w))
    return w


def gap_num(l: float, r: float, d: float) -> int:
    return lib().jvo_gap_num(l, r, d)


def cpml_ab(c: int, n: int, m: int, vp: float, delta: float, fm: float, dt: float):
    out = np.zeros(4, np.float64)
    active = lib().jvo_cpml_ab(c, n, m, vp, delta, fm, dt, _d(out))
    return bool(active), out


def n_inside_receivers(p: Problem) -> int:
    pc = p._c()
    return lib().jvo_select_inside(C.byref(pc), pc.recv_xyz, pc.n_recv, None)


def forward(p: Problem, shot: int = 0, precision: str = "f64"):
    """Traces (vx, vy, vz), each [n_recv_inside, nt] float64."""
    L = lib(precision)
    pc = p._c()
    nt = L.jvo_ntime(p.T, p.dt)
    nr = L.jvo_select_inside(C.byref(pc), pc.recv_xyz, pc.n_recv, None)
    vp, vs, rho = p._model()
    out = [np.zeros((max(nr, 1), nt), np.float64) for _ in range(3)]
    rc = L.jvo_forward(C.byref(pc), _f(vp), _f(vs), _f(rho), shot, _d(out[0]), _d(out[1]), _d(out[2]))
    if rc != 0:
        raise RuntimeError(f"jvo_forward failed: {rc}")
    return tuple(o[:nr] for o in out)


def rtm_shot(p: Problem, obs, shot: int = 0, images=None, precision: str = "f64", want_recon: bool = False):
    """Stack one shot into images (dict ip, pp, ps, sp, ss of gridphy FP64)."""
    L = lib(precision)
    pc = p._c()
    nt = L.jvo_ntime(p.T, p.dt)
    shape = (p.nz, p.ny, p.nx)
    if images is None:
        images = {k: np.zeros(shape, np.float64) for k in ("ip", "pp", "ps", "sp", "ss")}
    vp, vs, rho = p._model()
    o = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1, nt) if a.size else np.zeros((1, nt)) for a in obs]
    err = C.c_double(-1.0)
    rc = L.jvo_rtm_shot(C.byref(pc), _f(vp), _f(vs), _f(rho), shot, _d(o[0]), _d(o[1]), _d(o[2]),
                        _d(images["ip"]), _d(images["pp"]), _d(images["ps"]), _d(images["sp"]),
                        _d(images["ss"]), C.byref(err) if want_recon else None)
    if rc != 0:
        raise RuntimeError(f"jvo_rtm_shot failed: {rc}")
    if want_recon:
        return images, err.value
    return images


def finalize_image(images: dict, nx: int, ny: int, nz: int):
    """Laplacian of the uncompensated images, then source compensation.

    Returns (compensated dict, laplacian dict); inputs are not modified."""
    comp = {k: np.array(v, dtype=np.float64, copy=True) for k, v in images.items()}
    lap = {k: np.zeros_like(comp[k]) for k in ("pp", "ps", "sp", "ss")}
    lib().jvo_finalize_image(nx, ny, nz, _d(comp["ip"]), _d(comp["pp"]), _d(comp["ps"]), _d(comp["sp"]),
                             _d(comp["ss"]), _d(lap["pp"]), _d(lap["ps"]), _d(lap["sp"]), _d(lap["ss"]))
    return comp, lap


class store16:
    """Context manager of the storage-precision study (jvo_set_store16):
    inside it, the `precision` library rounds every stored wavefield
    component to FP16 ("fp16") or BF16 ("bf16") after each update, with a
    power-of-two scale per z plane; on exit storage is plain again.  The
    setting is process-wide state of that library."""

    def __init__(self, kind: str, precision: str = "f32"):
        self.mode = {"f32": 0, "fp16": 1, "bf16": 2}[kind]
        self.precision = precision

    def __enter__(self):
        lib(self.precision).jvo_set_store16(self.mode)
        return self

    def __exit__(self, *exc):
        lib(self.precision).jvo_set_store16(0)
        return False


def rtm_sample(p: Problem, steps: int, shot: int = 0) -> float:
    """Runs `steps` steps of every propagation of one RTM shot; returns
    the number of cell-updates performed."""
    L = lib("f64")
    pc = p._c()
    vp, vs, rho = p._model()
    r = L.jvo_rtm_sample(C.byref(pc), _f(vp), _f(vs), _f(rho), shot, steps)
    if r < 0:
        raise RuntimeError("jvo_rtm_sample failed")
    return r
