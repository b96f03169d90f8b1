"""jv -- single-B200 elastic FDTD modelling and VOWR RTM (Python front end).

This package is the Python mirror of the reference's modelling/RTM calls
(jarvis ``fdtd3d_blend_elastic_model_mpi`` / ``rtm3d_blend_model_mpi_module``)
over the C ABI of ``libjv.so`` (include/jv/jv.h).  All computation runs in
the CUDA library; there is no CPU fallback: importing works anywhere, but
creating a context raises ``JvError`` when libjv.so is missing or no CUDA
device is usable.

Typical use::

    jv = importlib.import_module("domain-decomposition-release_b200")
    s = jv.synth.small_case()
    with jv.Context.from_survey(s) as ctx:
        vx, vy, vz = ctx.forward(0)
        ctx.rtm_shot(0, (vx, vy, vz))
        img = ctx.finalize()
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import project, synth  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libjv.so")

JV_OK, JV_EINVAL, JV_ENOMEM, JV_ECUDA, JV_EIO, JV_ETIMEOUT, JV_ECANCELED, JV_ESTATE, JV_ENOTSUP = (
    0, -1, -2, -3, -4, -5, -6, -7, -8)
JV_FP32, JV_BF16, JV_FP16 = 0, 1, 2
JV_STORE_AUTO, JV_STORE_DEVICE, JV_STORE_HOST = 0, 1, 2
IMG_IP, IMG_PP, IMG_PS, IMG_SP, IMG_SS = range(5)

# every symbol include/jv/jv.h declares
EXPORTS = (
    "jv_options_default", "jv_create", "jv_open", "jv_set_geometry", "jv_set_model", "jv_get_info",
    "jv_get_kernel_config",
    "jv_reconstruction_energy",
    "jv_forward",
    "jv_forward_device", "jv_rtm_shot", "jv_rtm_shot_device", "jv_image_reset", "jv_image_get",
    "jv_image_finalize", "jv_image_get_device", "jv_run_project", "jv_set_profiling", "jv_profile_entry",
    "jv_last_timing", "jv_sync", "jv_close", "jv_last_error", "jv_build_info", "jv_forward_noalloc",
    "jv_image_set", "jv_image_set_device", "jv_run_project_shard", "jv_read_argfile", "jv_rtm_batch",
    "jv_submit", "jv_poll", "jv_wait", "jv_cancel",
    "jv_footprint", "jv_server_create", "jv_server_submit", "jv_server_poll", "jv_server_wait", "jv_server_cancel",
    "jv_server_get_stats", "jv_server_close", "jv_frame_make", "jv_fld_write", "jv_fld_read", "jv_raw_read",
    "jv_rtm_forward_pass", "jv_rtm_reverse_begin", "jv_rtm_reverse_op", "jv_rtm_reverse_end", "jv_stream_probe",
)
(OP_INJECT_RECEIVERS, OP_BACKWARD_STRESS, OP_REVERSE_VEL_PML, OP_REVERSE_VEL, OP_INJECT_BOUNDARY_STRESS,
 OP_BACKWARD_VEL_IMAGE, OP_REVERSE_STRESS_PML, OP_REVERSE_STRESS, OP_INJECT_BOUNDARY_VEL) = range(9)
JOB_FORWARD, JOB_RTM = 0, 1
JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_CANCELLED = 0, 1, 2, 3

REDUCE_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_double), C.c_size_t, C.c_void_p)


class JvError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"jv error {code}: {msg}")
        self.code = code


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("pml", C.c_int),
                ("dx", C.c_float), ("dy", C.c_float), ("dz", C.c_float)]


class Options(C.Structure):
    _fields_ = [("device", C.c_int), ("rec_width", C.c_int), ("precision", C.c_int), ("store_mode", C.c_int),
                ("use_graphs", C.c_int), ("graph_steps", C.c_int), ("store_budget", C.c_size_t),
                ("kernel_variant", C.c_int), ("zchunk", C.c_int), ("tile_gx", C.c_int), ("tile_gy", C.c_int),
                ("min_blocks", C.c_int), ("pml_min_blocks", C.c_int), ("planes_per_thread", C.c_int),
                ("pml_planes_per_thread", C.c_int), ("run_chunks", C.c_int), ("autotune", C.c_int)]


class Job(C.Structure):
    _fields_ = [("kind", C.c_int), ("shot", C.c_int), ("obs", C.POINTER(C.c_float) * 3),
                ("out", C.POINTER(C.c_float) * 3)]


class Request(C.Structure):
    _fields_ = [("kind", C.c_int), ("grid", Grid), ("vp", C.POINTER(C.c_float)), ("vs", C.POINTER(C.c_float)),
                ("rho", C.POINTER(C.c_float)), ("dt", C.c_float), ("fm", C.c_float), ("nt", C.c_int),
                ("rec_width", C.c_int), ("shot_xyz", C.c_float * 3), ("n_recv", C.c_int),
                ("recv_xyz", C.POINTER(C.c_float)), ("obs", C.POINTER(C.c_float) * 3),
                ("out", C.POINTER(C.c_float) * 3), ("image", C.POINTER(C.c_double) * 5),
                ("precision", C.c_int)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("failed", C.c_longlong),
                ("cancelled", C.c_longlong), ("running", C.c_longlong), ("queued", C.c_longlong),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double),
                ("bytes_in_use", C.c_size_t), ("budget", C.c_size_t), ("reused", C.c_longlong),
                ("pooled", C.c_longlong), ("device_ms", C.c_double)]


class ArgFileC(C.Structure):
    _fields_ = [("model_path", C.c_char * 1024), ("shot_path", C.c_char * 1024), ("rece_path", C.c_char * 1024),
                ("output_path", C.c_char * 1024), ("is_output", C.c_int), ("t_snap", C.c_int), ("pml_num", C.c_int),
                ("fm", C.c_float), ("dt", C.c_float), ("T", C.c_float), ("x_divide_num", C.c_int),
                ("y_divide_num", C.c_int), ("z_divide_num", C.c_int), ("slots_per_node", C.c_int),
                ("rec_width", C.c_int), ("vp_path", C.c_char * 1024), ("vs_path", C.c_char * 1024),
                ("rho_path", C.c_char * 1024), ("n_rows", C.c_int), ("n_cols", C.c_int), ("n_slices", C.c_int),
                ("d_rows", C.c_float), ("d_cols", C.c_float), ("d_slices", C.c_float), ("save_fld", C.c_int)]


class Frame(C.Structure):
    """The reference's Frame as it lies in memory (jv_frame; a .fld header)."""
    _fields_ = [("n_elem", C.c_uint64), ("n_rows", C.c_uint64), ("n_elem_slice", C.c_uint64),
                ("n_cols", C.c_uint32), ("n_slices", C.c_uint32),
                ("d_rows", C.c_float), ("d_cols", C.c_float), ("d_slices", C.c_float),
                ("l_rows", C.c_float), ("l_cols", C.c_float), ("l_slices", C.c_float),
                ("r_rows", C.c_float), ("r_cols", C.c_float), ("r_slices", C.c_float), ("type", C.c_int32)]


def make_frame(n_rows, n_cols=1, n_slices=1, d=(0.0, 0.0, 0.0), l=(0.0, 0.0, 0.0)) -> Frame:
    f = Frame()
    lib().jv_frame_make(n_rows, n_cols, n_slices, d[0], d[1], d[2], l[0], l[1], l[2], C.byref(f))
    return f


def fld_write(path_noext: str, frame: Frame, data: np.ndarray) -> str:
    """Field::save(.., binary_fld) through libjv: path_noext + '.fld'."""
    a = np.ascontiguousarray(data, dtype=np.float32)
    if a.size != frame.n_elem:
        raise JvError(JV_EINVAL, "data size does not match the frame")
    _check(lib().jv_fld_write(path_noext.encode(), C.byref(frame), _fptr(a)))
    return path_noext + ".fld"


def fld_read(path: str):
    """(Frame, float32 array (n_slices, n_cols, n_rows)) of a .fld file."""
    f = Frame()
    _check(lib().jv_fld_read(path.encode(), C.byref(f), None, 0))
    a = np.empty(int(f.n_elem), np.float32)
    _check(lib().jv_fld_read(path.encode(), C.byref(f), _fptr(a), a.size))
    return f, a.reshape(int(f.n_slices), int(f.n_cols), int(f.n_rows))


def read_argfile(proj_path: str) -> dict:
    """The project's argfile as libjv reads it (jv_read_argfile)."""
    a = ArgFileC()
    _check(lib().jv_read_argfile(proj_path.encode(), C.byref(a)))
    out = {}
    for name, _ in ArgFileC._fields_:
        v = getattr(a, name)
        out[name] = v.decode() if isinstance(v, bytes) else v
    return out


class Info(C.Structure):
    _fields_ = [("grid", Grid), ("nt", C.c_int), ("n_shot", C.c_int), ("n_recv", C.c_int),
                ("rec_width", C.c_int), ("precision", C.c_int), ("n_ext", C.c_longlong),
                ("n_phy", C.c_longlong), ("store_bytes_per_step", C.c_size_t), ("device_bytes", C.c_size_t),
                ("store_on_device", C.c_int)]


_lib = None


def build(force: bool = False) -> str:
    """Compiles libjv.so for sm_100a in-tree (nvcc; no GPU needed)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-s", "-C", os.path.join(HERE, "csrc"), "-j8"], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    """Loads libjv.so (raising JvError if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise JvError(JV_ENOTSUP, f"{LIB_PATH} is not built (run build())")
    L = C.CDLL(LIB_PATH)
    fp, dp, vp = C.POINTER(C.c_float), C.POINTER(C.c_double), C.c_void_p
    ctxp = C.c_void_p
    L.jv_options_default.argtypes = [C.POINTER(Options)]
    L.jv_options_default.restype = None
    L.jv_create.argtypes = [C.POINTER(Grid), fp, fp, fp, C.c_float, C.c_float, C.c_int, C.POINTER(Options),
                            C.POINTER(ctxp)]
    L.jv_open.argtypes = [C.c_char_p, C.POINTER(Options), C.POINTER(ctxp)]
    L.jv_set_geometry.argtypes = [ctxp, C.c_int, fp, C.c_int, fp]
    L.jv_set_model.argtypes = [ctxp, fp, fp, fp]
    L.jv_get_info.argtypes = [ctxp, C.POINTER(Info)]
    L.jv_get_kernel_config.argtypes = [ctxp, C.POINTER(Options)]
    L.jv_reconstruction_energy.argtypes = [ctxp, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.jv_forward.argtypes = [ctxp, C.c_int, fp, fp, fp]
    L.jv_forward_device.argtypes = [ctxp, C.c_int, vp, vp, vp]
    L.jv_rtm_shot.argtypes = [ctxp, C.c_int, fp, fp, fp]
    L.jv_rtm_shot_device.argtypes = [ctxp, C.c_int, vp, vp, vp]
    L.jv_image_reset.argtypes = [ctxp]
    L.jv_image_get.argtypes = [ctxp, C.c_int, dp]
    L.jv_image_finalize.argtypes = [ctxp] + [fp] * 8
    L.jv_image_get_device.argtypes = [ctxp, C.c_int, vp]
    L.jv_image_set.argtypes = [ctxp, C.c_int, dp]
    L.jv_image_set_device.argtypes = [ctxp, C.c_int, vp]
    L.jv_set_profiling.argtypes = [ctxp, C.c_int]
    L.jv_profile_entry.argtypes = [ctxp, C.c_int, C.POINTER(C.c_char_p), dp, C.POINTER(C.c_longlong)]
    L.jv_run_project.argtypes = [ctxp]
    L.jv_rtm_batch.argtypes = [ctxp, C.c_int, C.POINTER(C.c_int), C.POINTER(fp)]
    L.jv_submit.argtypes = [ctxp, C.POINTER(Job), C.POINTER(C.c_longlong)]
    L.jv_poll.argtypes = [ctxp, C.c_longlong, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.jv_wait.argtypes = [ctxp, C.c_longlong, C.c_double, C.POINTER(C.c_int)]
    L.jv_cancel.argtypes = [ctxp, C.c_longlong]
    L.jv_footprint.argtypes = [C.POINTER(Grid), C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_size_t)]
    L.jv_server_create.argtypes = [C.c_int, C.c_int, C.c_size_t, C.POINTER(vp)]
    L.jv_server_submit.argtypes = [vp, C.POINTER(Request), C.POINTER(C.c_longlong)]
    L.jv_server_poll.argtypes = [vp, C.c_longlong, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.jv_server_wait.argtypes = [vp, C.c_longlong, C.c_double, C.POINTER(C.c_int)]
    L.jv_server_cancel.argtypes = [vp, C.c_longlong]
    L.jv_server_get_stats.argtypes = [vp, C.POINTER(ServerStats)]
    L.jv_server_close.argtypes = [vp]
    L.jv_run_project_shard.argtypes = [ctxp, C.c_int, C.c_int, REDUCE_FN, C.c_void_p]
    L.jv_read_argfile.argtypes = [C.c_char_p, C.POINTER(ArgFileC)]
    L.jv_forward_noalloc.argtypes = [C.POINTER(Grid), vp, vp, vp, C.c_float, C.c_float, C.c_int, fp, C.c_int, fp,
                                     vp, vp, vp, C.POINTER(C.c_int), vp]
    L.jv_frame_make.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32] + [C.c_float] * 6 + [C.POINTER(Frame)]
    L.jv_frame_make.restype = None
    L.jv_fld_write.argtypes = [C.c_char_p, C.POINTER(Frame), fp]
    L.jv_fld_read.argtypes = [C.c_char_p, C.POINTER(Frame), fp, C.c_size_t]
    L.jv_raw_read.argtypes = [C.c_char_p, C.c_size_t, fp]
    L.jv_rtm_forward_pass.argtypes = [ctxp, C.c_int]
    L.jv_rtm_reverse_begin.argtypes = [ctxp, C.c_int, vp, vp, vp]
    L.jv_rtm_reverse_op.argtypes = [ctxp, C.c_int, C.c_int]
    L.jv_rtm_reverse_end.argtypes = [ctxp]
    L.jv_last_timing.argtypes = [ctxp, dp]
    L.jv_stream_probe.argtypes = [C.c_int, C.c_int, C.c_int, C.c_size_t, C.c_int, dp]
    L.jv_sync.argtypes = [ctxp]
    L.jv_close.argtypes = [ctxp]
    L.jv_last_error.argtypes = []
    L.jv_last_error.restype = C.c_char_p
    L.jv_build_info.argtypes = []
    L.jv_build_info.restype = C.c_char_p
    for n in EXPORTS:
        if n not in ("jv_options_default", "jv_last_error", "jv_build_info", "jv_frame_make"):
            getattr(L, n).restype = C.c_int
    _lib = L
    return L


def _check(rc: int) -> None:
    if rc != JV_OK:
        msg = lib().jv_last_error().decode(errors="replace")
        raise JvError(rc, msg)


def _fptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_float)) if a is not None else None


def default_options(**kw) -> Options:
    o = Options()
    lib().jv_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Context:
    """One problem resident on one GPU (a jv_ctx)."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    # -- construction -----------------------------------------------------
    @classmethod
    def create(cls, nx, ny, nz, pml, dx, dy, dz, vp, vs, rho, dt, fm, nt, **opts) -> "Context":
        L = lib()
        g = Grid(nx, ny, nz, pml, dx, dy, dz)
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (vp, vs, rho)]
        for a in arrs:
            if a.size != nx * ny * nz:
                raise JvError(JV_EINVAL, "model array size does not match the grid")
        o = default_options(**opts)
        h = C.c_void_p()
        _check(L.jv_create(C.byref(g), _fptr(arrs[0]), _fptr(arrs[1]), _fptr(arrs[2]), dt, fm, int(nt), C.byref(o),
                           C.byref(h)))
        return cls(h)

    @classmethod
    def from_survey(cls, s, **opts) -> "Context":
        opts.setdefault("rec_width", s.rec_width)
        c = cls.create(s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.vp, s.vs, s.rho, s.dt, s.fm, s.nt, **opts)
        c.set_geometry(s.shots, s.recvs)
        return c

    @classmethod
    def open(cls, proj_path: str, **opts) -> "Context":
        """Reads a reference project directory (argfile.json + geometry + .gms)."""
        L = lib()
        o = default_options(**opts)
        h = C.c_void_p()
        _check(L.jv_open(proj_path.encode(), C.byref(o), C.byref(h)))
        return cls(h)

    def set_geometry(self, shots, recvs) -> None:
        sh = np.ascontiguousarray(shots, dtype=np.float32).reshape(-1, 3)
        rc = np.ascontiguousarray(recvs, dtype=np.float32).reshape(-1, 3)
        _check(lib().jv_set_geometry(self._h, sh.shape[0], _fptr(sh), rc.shape[0], _fptr(rc)))

    def set_model(self, vp, vs, rho) -> None:
        """A new model of the same grid (jv_set_model): buffers and captured
        graphs are kept."""
        i = self.info()
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (vp, vs, rho)]
        for a in arrs:
            if a.size != i.grid.nx * i.grid.ny * i.grid.nz:
                raise JvError(JV_EINVAL, "model array size does not match the grid")
        _check(lib().jv_set_model(self._h, _fptr(arrs[0]), _fptr(arrs[1]), _fptr(arrs[2])))

    # -- queries ------------------------------------------------------------
    def reconstruction_energy(self):
        """(energy at the end of the last RTM shot's forward pass, energy left
        after its reconstruction back to t = 0), FP64."""
        a, b = C.c_double(), C.c_double()
        _check(lib().jv_reconstruction_energy(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def kernel_config(self) -> dict:
        """The options this context runs with, the kernel choice as made."""
        o = Options()
        _check(lib().jv_get_kernel_config(self._h, C.byref(o)))
        return {k: getattr(o, k) for k, _ in Options._fields_}

    def info(self) -> Info:
        i = Info()
        _check(lib().jv_get_info(self._h, C.byref(i)))
        return i

    def last_ms(self) -> float:
        v = C.c_double()
        _check(lib().jv_last_timing(self._h, C.byref(v)))
        return v.value

    # -- modelling / migration ---------------------------------------------
    def forward(self, shot: int):
        """Traces (vx, vy, vz), each float32 [n_recv, nt] (host arrays)."""
        i = self.info()
        out = [np.zeros((i.n_recv, i.nt), np.float32) for _ in range(3)]
        _check(lib().jv_forward(self._h, shot, _fptr(out[0]), _fptr(out[1]), _fptr(out[2])))
        return tuple(out)

    def forward_device(self, shot: int, ptrs) -> None:
        """Device-pointer variant: ptrs = 3 device addresses (ints)."""
        _check(lib().jv_forward_device(self._h, shot, *[C.c_void_p(int(p)) if p else None for p in ptrs]))

    def rtm_shot(self, shot: int, obs) -> None:
        o = [np.ascontiguousarray(a, dtype=np.float32) for a in obs]
        _check(lib().jv_rtm_shot(self._h, shot, _fptr(o[0]), _fptr(o[1]), _fptr(o[2])))

    def rtm_shot_device(self, shot: int, ptrs) -> None:
        _check(lib().jv_rtm_shot_device(self._h, shot, *[C.c_void_p(int(p)) for p in ptrs]))

    def image_reset(self) -> None:
        _check(lib().jv_image_reset(self._h))

    def image(self, kind: int) -> np.ndarray:
        i = self.info()
        out = np.zeros((i.grid.nz, i.grid.ny, i.grid.nx), np.float64)
        _check(lib().jv_image_get(self._h, kind, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def images(self) -> dict:
        return {k: self.image(v) for k, v in (("ip", IMG_IP), ("pp", IMG_PP), ("ps", IMG_PS), ("sp", IMG_SP),
                                              ("ss", IMG_SS))}

    def finalize(self, out=None):
        """(compensated {pp,ps,sp,ss}, laplacian {pp,ps,sp,ss}) float32.  out:
        eight C-contiguous float32 arrays of gridphy to fill (e.g. views of
        pinned memory, reused across shots); None allocates them."""
        i = self.info()
        shp = (i.grid.nz, i.grid.ny, i.grid.nx)
        if out is None:
            arr = [np.zeros(shp, np.float32) for _ in range(8)]
        else:
            arr = list(out)
            if len(arr) != 8 or any(a.dtype != np.float32 or not a.flags.c_contiguous or a.size != i.n_phy
                                    for a in arr):
                raise JvError(JV_EINVAL, "finalize(out=...) takes eight C-contiguous float32 arrays of gridphy")
        _check(lib().jv_image_finalize(self._h, *[_fptr(a) for a in arr]))
        keys = ("pp", "ps", "sp", "ss")
        return dict(zip(keys, arr[:4])), dict(zip(keys, arr[4:]))

    def image_to_device(self, kind: int, dev_ptr: int) -> None:
        """Copies one FP64 accumulator into device memory at dev_ptr."""
        _check(lib().jv_image_get_device(self._h, kind, C.c_void_p(int(dev_ptr))))

    def set_image(self, kind: int, arr: np.ndarray) -> None:
        """Overwrites one FP64 accumulator from a host array of gridphy."""
        i = self.info()
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.size != i.n_phy:
            raise JvError(JV_EINVAL, f"image has {a.size} values, gridphy has {i.n_phy}")
        _check(lib().jv_image_set(self._h, kind, a.ctypes.data_as(C.POINTER(C.c_double))))

    def image_from_device(self, kind: int, dev_ptr: int) -> None:
        """Overwrites one FP64 accumulator from device memory at dev_ptr."""
        _check(lib().jv_image_set_device(self._h, kind, C.c_void_p(int(dev_ptr))))

    def set_profiling(self, on: bool) -> None:
        _check(lib().jv_set_profiling(self._h, 1 if on else 0))

    def profile(self) -> dict:
        """{kernel name: (total ms, launches)} since profiling was switched on."""
        out, i = {}, 0
        L = lib()
        while True:
            nm, ms, n = C.c_char_p(), C.c_double(), C.c_longlong()
            if L.jv_profile_entry(self._h, i, C.byref(nm), C.byref(ms), C.byref(n)) != JV_OK:
                break
            out[nm.value.decode()] = (ms.value, n.value)
            i += 1
        return out

    def run_project(self) -> None:
        _check(lib().jv_run_project(self._h))

    def rtm_batch(self, shots, obs) -> None:
        """jv_rtm_batch: obs[k] = (vx, vy, vz) float32 host arrays of shots[k]."""
        n = len(shots)
        keep = [np.ascontiguousarray(a, dtype=np.float32) for o in obs for a in o]
        ptrs = (C.POINTER(C.c_float) * (3 * n))(*[_fptr(a) for a in keep])
        sh = (C.c_int * n)(*[int(s) for s in shots])
        _check(lib().jv_rtm_batch(self._h, n, sh, ptrs))

    def submit(self, kind: int, shot: int, obs=None, out=None) -> int:
        """jv_submit; the arrays in obs / out must live until the job ends
        (this object keeps references to them)."""
        j = Job()
        j.kind, j.shot = kind, shot
        refs = []
        for q in range(3):
            if obs is not None:
                a = np.ascontiguousarray(obs[q], dtype=np.float32)
                refs.append(a)
                j.obs[q] = _fptr(a)
            if out is not None and out[q] is not None:
                if out[q].dtype != np.float32 or not out[q].flags.c_contiguous:
                    raise JvError(JV_EINVAL, "job outputs must be C-contiguous float32 arrays")
                refs.append(out[q])
                j.out[q] = _fptr(out[q])
        jid = C.c_longlong()
        _check(lib().jv_submit(self._h, C.byref(j), C.byref(jid)))
        self._job_refs = getattr(self, "_job_refs", {})
        self._job_refs[jid.value] = refs
        return jid.value

    def poll(self, jid: int):
        """(state, result) of a job."""
        st, res = C.c_int(), C.c_int()
        _check(lib().jv_poll(self._h, jid, C.byref(st), C.byref(res)))
        if st.value in (JOB_DONE, JOB_CANCELLED):
            getattr(self, "_job_refs", {}).pop(jid, None)
        return st.value, res.value

    def wait(self, jid: int, timeout: float = -1.0) -> int:
        """Waits for a job; returns its result (JvError on JV_ETIMEOUT)."""
        res = C.c_int()
        _check(lib().jv_wait(self._h, jid, timeout, C.byref(res)))
        getattr(self, "_job_refs", {}).pop(jid, None)
        return res.value

    def cancel(self, jid: int) -> None:
        _check(lib().jv_cancel(self._h, jid))

    def run_project_shard(self, rank: int, world: int, reduce=None) -> None:
        """jv_run_project_shard; `reduce(arr)` sums a float64 numpy array in
        place over the job's ranks."""
        if reduce is None:
            cb = C.cast(None, REDUCE_FN)
        else:
            def _cb(ptr, n, _user):
                try:
                    reduce(np.ctypeslib.as_array(ptr, shape=(n,)))
                    return 0
                except Exception:  # reported to the library as a failed reduce
                    return 1
            cb = REDUCE_FN(_cb)
        _check(lib().jv_run_project_shard(self._h, rank, world, cb, None))

    def sync(self) -> None:
        _check(lib().jv_sync(self._h))

    def close(self) -> None:
        if self._h:
            lib().jv_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def stream_probe(n_read: int, n_write: int, n: int, reps: int = 5, device: int = 0) -> float:
    """GB/s of a pointwise pass over n_read + n_write arrays of n floats
    (jv_stream_probe): the attainable bandwidth of a kernel with that
    footprint."""
    g = C.c_double()
    _check(lib().jv_stream_probe(device, n_read, n_write, n, reps, C.byref(g)))
    return g.value


def footprint(nx, ny, nz, pml, nt, rec_width=1, kind=JOB_RTM, n_recv=0) -> int:
    """Device bytes a context holds for one request of this size (jv_footprint)."""
    g = Grid(nx, ny, nz, pml, 1.0, 1.0, 1.0)
    b = C.c_size_t()
    _check(lib().jv_footprint(C.byref(g), nt, rec_width, kind, n_recv, C.byref(b)))
    return b.value


class Server:
    """jv_server: requests of their own size and model, admitted into
    `slots` concurrent workers under an HBM budget (bytes; 0 = 90 % of the
    free device memory)."""

    def __init__(self, slots: int = 4, budget: int = 0, device: int = 0):
        h = C.c_void_p()
        _check(lib().jv_server_create(device, slots, budget, C.byref(h)))
        self._h = h
        self._refs = {}

    def submit(self, kind, nx, ny, nz, pml, dx, dy, dz, vp, vs, rho, dt, fm, nt, shot_xyz, recv_xyz,
               rec_width=1, obs=None, out=None, image=None, precision=JV_FP32) -> int:
        """Queues one request.  out (FORWARD) / obs (RTM) are 3 float32
        arrays [n_kept][nt]; image (RTM) up to 5 float64 arrays of gridphy
        (ip, pp, ps, sp, ss; None skips one); precision: the RTM boundary
        store's (JV_FP32, JV_BF16, JV_FP16).  The arrays are kept alive here
        until the request has been waited for."""
        r = Request()
        r.kind = kind
        r.precision = precision
        r.grid = Grid(nx, ny, nz, pml, dx, dy, dz)
        refs = []

        def f32(a):
            a = np.ascontiguousarray(a, dtype=np.float32)
            refs.append(a)
            return _fptr(a)

        r.vp, r.vs, r.rho = f32(vp), f32(vs), f32(rho)
        r.dt, r.fm, r.nt, r.rec_width = dt, fm, nt, rec_width
        for q in range(3):
            r.shot_xyz[q] = float(shot_xyz[q])
        rv = np.ascontiguousarray(recv_xyz, dtype=np.float32).reshape(-1, 3)
        refs.append(rv)
        r.n_recv = rv.shape[0]
        r.recv_xyz = _fptr(rv)
        for q in range(3):
            if obs is not None:
                r.obs[q] = f32(obs[q])
            if out is not None and out[q] is not None:
                if out[q].dtype != np.float32 or not out[q].flags.c_contiguous:
                    raise JvError(JV_EINVAL, "request outputs must be C-contiguous float32 arrays")
                refs.append(out[q])
                r.out[q] = _fptr(out[q])
        if image is not None:
            for q in range(5):
                if image[q] is not None:
                    if image[q].dtype != np.float64 or not image[q].flags.c_contiguous:
                        raise JvError(JV_EINVAL, "request images must be C-contiguous float64 arrays")
                    refs.append(image[q])
                    r.image[q] = image[q].ctypes.data_as(C.POINTER(C.c_double))
        rid = C.c_longlong()
        _check(lib().jv_server_submit(self._h, C.byref(r), C.byref(rid)))
        self._refs[rid.value] = refs
        return rid.value

    def submit_survey(self, kind, s, shot: int = 0, obs=None, precision=JV_FP32, outs=None):
        """Queues shot `shot` of a synth.Survey-like object; returns (id,
        outputs): the three trace arrays [n_recv][nt] of a FORWARD request,
        or the five image arrays (ip, pp, ps, sp, ss; gridphy, float64) of an
        RTM request, filled when the request is done.  outs: those arrays,
        allocated by the caller (e.g. reused), instead of new ones."""
        rv = np.ascontiguousarray(s.recvs, dtype=np.float32).reshape(-1, 3)
        if outs is not None:
            want = (np.float32, (rv.shape[0], s.nt), 3) if kind == JOB_FORWARD else (np.float64, (s.nz, s.ny, s.nx), 5)
            outs = tuple(outs)
            if len(outs) != want[2] or any(o.dtype != want[0] or o.shape != want[1] or not o.flags.c_contiguous
                                           for o in outs):
                raise JvError(JV_EINVAL, "outs do not match the request's outputs")
            rid = self.submit(kind, s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.vp, s.vs, s.rho, s.dt, s.fm, s.nt,
                              s.shots[shot], rv, rec_width=s.rec_width, obs=obs,
                              **({"out": outs} if kind == JOB_FORWARD else {"image": outs, "precision": precision}))
            return rid, outs
        if kind == JOB_FORWARD:
            outs = tuple(np.zeros((rv.shape[0], s.nt), np.float32) for _ in range(3))
            rid = self.submit(kind, s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.vp, s.vs, s.rho, s.dt, s.fm, s.nt,
                              s.shots[shot], rv, rec_width=s.rec_width, out=outs)
        else:
            outs = tuple(np.zeros((s.nz, s.ny, s.nx), np.float64) for _ in range(5))
            rid = self.submit(kind, s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.vp, s.vs, s.rho, s.dt, s.fm, s.nt,
                              s.shots[shot], rv, rec_width=s.rec_width, obs=obs, image=outs, precision=precision)
        return rid, outs

    def poll(self, rid: int):
        st, res = C.c_int(), C.c_int()
        _check(lib().jv_server_poll(self._h, rid, C.byref(st), C.byref(res)))
        return st.value, res.value

    def wait(self, rid: int, timeout: float = -1.0) -> int:
        res = C.c_int()
        _check(lib().jv_server_wait(self._h, rid, timeout, C.byref(res)))
        self._refs.pop(rid, None)
        return res.value

    def cancel(self, rid: int) -> None:
        _check(lib().jv_server_cancel(self._h, rid))

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().jv_server_get_stats(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_}

    def close(self) -> None:
        if self._h:
            lib().jv_server_close(self._h)
            self._h = None
            self._refs.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
