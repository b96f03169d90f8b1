"""Project files in the reference's formats.

* argfile.json -- JSON with ``//`` comments, keys of ArgList
  (src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/
  elastic_1_fdtd3d_model_mpi/fdtd3d_0_base_module/fdtd3d_base_1_interface.hpp:
  27-113).  Paths are prefixed with the project directory, exactly as the
  reference does; unknown keys are ignored and the optional keys this
  library adds (``rec_width``, ``precision``) default to the reference
  behaviour.
* shot.txt / rece.txt -- a count, then ``x y z`` per line in metres
  (src/jarvis_cpp/jarvis/.jarvis_1_util/.jarvis_2_geometry/
  jarvis_device_geometry_meat.hpp:6-54).
* .gms models -- 240-byte header, then per parameter a 64-byte name and the
  data with z fastest, then x, then y (src/jarvis_cpp/jarvis/.jarvis_1_util/
  .jarvis_0_gms/jarvis_device_gms_meat.hpp:11-79).  Parameters in order
  vp, vs, rho.
* raw models -- one float32 file per parameter (vp, vs, rho), x fastest, on
  a Frame the argfile gives (optional keys vp_path, vs_path, rho_path,
  n_rows, n_cols, n_slices, d_rows, d_cols, d_slices), in place of the
  reference's edit of its loader to call Field::read_raw
  (src/jarvis_cpp/jarvis/.jarvis_0_meta/.jarvis_2_field/
  jarvis_1_host_field_meat.hpp:65-79; README.md:131-144).
* .fld -- the reference Frame struct's 72 bytes, then the float32 data
  (save_as_binary_fld, jarvis_1_host_field_meat.hpp:81-89).
* traces -- ``%10.6e\t`` per sample, one line per receiver
  (src/jarvis_cpp/jarvis/.jarvis_0_meta/.jarvis_2_field/
  jarvis_1_host_field_meat.hpp:159-197); images -- raw float32, x fastest,
  file name suffix ``_{nx}_{ny}_{nz}_{lx}_{ly}_{lz}.raw`` (Frame::size_info,
  jarvis_0_frame_meat.hpp:347-351).
"""
from __future__ import annotations

import json
import os
import re
import struct

import numpy as np

GMS_HEADER = struct.Struct("<h64sh6bh3f3I3f127sx")
assert GMS_HEADER.size == 240

ARG_KEYS_STR = ("model_path", "shot_path", "rece_path", "output_path")
ARG_KEYS_INT = ("x_divide_num", "y_divide_num", "z_divide_num", "slots_per_node", "pml_num", "t_snap")
ARG_KEYS_FLOAT = ("fm", "T", "dt")


def strip_json_comments(text: str) -> str:
    """Removes // line comments and /* */ block comments outside strings."""
    out, i, n, in_str = [], 0, len(text), False
    while i < n:
        c = text[i]
        if in_str:
            out.append(c)
            if c == "\\" and i + 1 < n:
                out.append(text[i + 1])
                i += 2
                continue
            if c == '"':
                in_str = False
            i += 1
            continue
        if c == '"':
            in_str = True
            out.append(c)
            i += 1
        elif text.startswith("//", i):
            j = text.find("\n", i)
            i = n if j < 0 else j
        elif text.startswith("/*", i):
            j = text.find("*/", i + 2)
            i = n if j < 0 else j + 2
        else:
            out.append(c)
            i += 1
    return "".join(out)


def read_argfile(proj_path: str) -> dict:
    """ArgList::mpi_read_arg_file semantics: proj_path + 'argfile.json';
    path values are prefixed with proj_path (string concatenation)."""
    if not proj_path.endswith("/"):
        proj_path = proj_path + "/"
    with open(proj_path + "argfile.json", "r") as f:
        raw = json.loads(strip_json_comments(f.read()))
    a = {"proj_path": proj_path}
    for k in ARG_KEYS_STR:
        a[k] = proj_path + str(raw.get(k, ""))
    for k in ARG_KEYS_INT:
        a[k] = int(raw.get(k, 0))
    for k in ARG_KEYS_FLOAT:
        a[k] = float(np.float32(raw.get(k, 0.0)))
    a["is_output"] = bool(raw.get("is_output", False))
    a["rec_width"] = int(raw.get("rec_width", 1))
    a["precision"] = str(raw.get("precision", "fp32"))
    return a


def write_argfile(proj_path: str, *, model_path: str, pml_num: int, fm: float, dt: float, T: float,
                  rec_width: int | None = None, extra: dict | None = None) -> None:
    lines = [
        "{",
        f'    "model_path": "{model_path}",',
        '    "shot_path": "shot.txt",',
        '    "rece_path": "rece.txt",',
        '    "output_path": "out/",',
        "    //",
        '    "is_output": false,',
        "    //",
        f'    "pml_num": {int(pml_num)},',
        f'    "fm": {repr(float(fm))},',
        f'    "dt": {repr(float(dt))},',
        f'    "T": {repr(float(T))},',
        '    "t_snap": -1,',
        "    //*mpi parameter: one subdomain",
        '    "x_divide_num": 1,',
        '    "y_divide_num": 1,',
        '    "z_divide_num": 1,',
    ]
    tail = ['    "slots_per_node": 1']
    if rec_width is not None:
        tail[-1] += ","
        tail.append(f'    "rec_width": {int(rec_width)}')
    for k, v in (extra or {}).items():
        tail[-1] += ","
        tail.append(f"    {json.dumps(k)}: {json.dumps(v)}")
    os.makedirs(proj_path, exist_ok=True)
    with open(os.path.join(proj_path, "argfile.json"), "w") as f:
        f.write("\n".join(lines + tail) + "\n}\n")


def read_points(path: str) -> np.ndarray:
    """Geometry::read_shot_line / read_recv_line: count, then x y z."""
    with open(path, "r") as f:
        tok = f.read().split()
    if not tok:
        raise ValueError(f"{path}: empty geometry file")
    n = int(tok[0])
    vals = np.array([float(t) for t in tok[1:1 + 3 * n]], dtype=np.float32)
    if vals.size != 3 * n:
        raise ValueError(f"{path}: expected {n} points")
    return vals.reshape(n, 3)


def write_points(path: str, pts: np.ndarray) -> None:
    pts = np.asarray(pts, dtype=np.float32).reshape(-1, 3)
    with open(path, "w") as f:
        f.write(f"{pts.shape[0]}\n")
        for p in pts:
            f.write(f"{p[0]:.6g} {p[1]:.6g} {p[2]:.6g}\n")


def write_gms(path: str, params: dict, d=(1.0, 1.0, 1.0), l=(0.0, 0.0, 0.0), name: str = "model") -> None:
    """Writes (nz, ny, nx) float32 arrays in the GMS layout."""
    arrs = list(params.items())
    nz, ny, nx = arrs[0][1].shape
    hdr = GMS_HEADER.pack(1, name.encode()[:64].ljust(64, b"\0"), 2024, 1, 1, 0, 0, 0, 3, len(arrs),
                          float(l[0]), float(l[1]), float(l[2]), nx, ny, nz, float(d[0]), float(d[1]),
                          float(d[2]), b"\0" * 127)
    with open(path, "wb") as f:
        f.write(hdr)
        for pname, a in arrs:
            a = np.asarray(a, dtype=np.float32)
            if a.shape != (nz, ny, nx):
                raise ValueError("all GMS parameters must share one grid")
            f.write(pname.encode()[:64].ljust(64, b"\0"))
            # data[i*nz + j*nx*nz + k]: z fastest, then x, then y
            f.write(np.ascontiguousarray(a.transpose(1, 2, 0)).tobytes())


def read_gms(path: str):
    """Returns (dict name -> (nz, ny, nx) float32, grid dict)."""
    with open(path, "rb") as f:
        buf = f.read()
    h = GMS_HEADER.unpack_from(buf, 0)
    para_num = h[9]
    lx, ly, lz, nx, ny, nz, dx, dy, dz = h[10:19]
    n = nx * ny * nz
    out, off = {}, 240
    for p in range(para_num):
        nm = buf[off:off + 64].split(b"\0")[0].decode(errors="replace") or f"p{p}"
        off += 64
        a = np.frombuffer(buf, dtype=np.float32, count=n, offset=off)
        off += 4 * n
        out[nm if nm not in out else f"{nm}{p}"] = np.ascontiguousarray(a.reshape(ny, nx, nz).transpose(2, 0, 1))
    return out, {"nx": nx, "ny": ny, "nz": nz, "dx": dx, "dy": dy, "dz": dz, "lx": lx, "ly": ly, "lz": lz}


def write_project(proj_path: str, s, *, model_name: str = "model.gms", rec_width_key: bool = True,
                  raw_model: bool = False, save_fld: bool = False) -> None:
    """Writes argfile.json, shot.txt, rece.txt and the model of a
    synth.Survey into proj_path (creating proj_path/out/): a GMS file, or
    with raw_model three raw float32 files (vp.raw, vs.raw, rho.raw, x
    fastest) named by the raw-model keys.  save_fld asks jv_run_project to
    write the images as .fld too."""
    os.makedirs(os.path.join(proj_path, "out"), exist_ok=True)
    extra = {}
    if raw_model:
        for nm in ("vp", "vs", "rho"):
            np.ascontiguousarray(getattr(s, nm), dtype=np.float32).tofile(os.path.join(proj_path, nm + ".raw"))
            extra[nm + "_path"] = nm + ".raw"
        extra.update({"n_rows": s.nx, "n_cols": s.ny, "n_slices": s.nz, "d_rows": float(s.dx),
                      "d_cols": float(s.dy), "d_slices": float(s.dz)})
        model_name = ""
    else:
        write_gms(os.path.join(proj_path, model_name), {"vp": s.vp, "vs": s.vs, "rho": s.rho},
                  d=(s.dx, s.dy, s.dz))
    if save_fld:
        extra["save_fld"] = True
    write_points(os.path.join(proj_path, "shot.txt"), s.shots)
    write_points(os.path.join(proj_path, "rece.txt"), s.recvs)
    write_argfile(proj_path, model_path=model_name, pml_num=s.pml, fm=s.fm, dt=s.dt, T=s.T,
                  rec_width=s.rec_width if rec_width_key else None, extra=extra)


# Frame (jarvis_0_frame_bones.hpp:9-51) on x86-64: n_elem, n_rows,
# n_elem_slice (uint64), n_cols, n_slices (uint32), d/l/r of rows, cols,
# slices (float), type (enum, int32)
FRAME = struct.Struct("<QQQII9fi")
assert FRAME.size == 72


def frame(nx: int, ny: int = 1, nz: int = 1, d=(0.0, 0.0, 0.0), l=(0.0, 0.0, 0.0)) -> dict:
    """Frame(nx, ny, nz, d, l) with its derived members and type
    (jarvis_0_frame_meat.hpp:27-65, set_frame_type :219-241)."""
    f32 = np.float32
    d = [f32(v) for v in d]
    l = [f32(v) for v in l]
    n = (nx, ny, nz)
    r = [f32(l[a] + f32(n[a] - 1) * d[a]) if n[a] > 0 else f32(0.0) for a in range(3)]
    l = [l[a] if n[a] > 0 else f32(0.0) for a in range(3)]
    spaced = any(v > 0 for v in d)
    one = (nx == 1 and ny == 1) or (nx == 1 and nz == 1) or (ny == 1 and nz == 1)
    two = (nx > 1 and ny > 1 and nz == 1) or (nx > 1 and nz > 1 and ny == 1) or (ny > 1 and nz > 1 and nx == 1)
    three = nx > 1 and ny > 1 and nz > 1
    t = (10 if spaced else 1) if one else (20 if spaced else 2) if two else (30 if spaced else 3) if three else 0
    return {"n_elem": nx * ny * nz, "n_rows": nx, "n_elem_slice": nx * ny, "n_cols": ny, "n_slices": nz,
            "d": d, "l": l, "r": r, "type": t}


def write_fld(path_noext: str, a: np.ndarray, d=(0.0, 0.0, 0.0), l=(0.0, 0.0, 0.0)) -> str:
    """A (nz, ny, nx) float32 field as path_noext + '.fld'."""
    a = np.asarray(a, dtype=np.float32)
    nz, ny, nx = a.shape if a.ndim == 3 else (1, 1, a.size)
    f = frame(nx, ny, nz, d, l)
    path = path_noext + ".fld"
    with open(path, "wb") as fh:
        fh.write(FRAME.pack(f["n_elem"], f["n_rows"], f["n_elem_slice"], f["n_cols"], f["n_slices"], *f["d"], *f["l"],
                            *f["r"], f["type"]))
        fh.write(np.ascontiguousarray(a).tobytes())
    return path


def read_fld(path: str):
    """(frame dict, float32 array (n_slices, n_cols, n_rows)) of a .fld file."""
    with open(path, "rb") as fh:
        buf = fh.read()
    v = FRAME.unpack_from(buf, 0)
    f = {"n_elem": v[0], "n_rows": v[1], "n_elem_slice": v[2], "n_cols": v[3], "n_slices": v[4],
         "d": list(v[5:8]), "l": list(v[8:11]), "r": list(v[11:14]), "type": v[14]}
    if f["n_elem"] != f["n_rows"] * f["n_cols"] * f["n_slices"] or len(buf) != 72 + 4 * f["n_elem"]:
        raise ValueError(f"{path}: bad .fld header or size")
    a = np.frombuffer(buf, dtype=np.float32, count=f["n_elem"], offset=72)
    return f, a.reshape(f["n_slices"], f["n_cols"], f["n_rows"]).copy()


def size_info(nx: int, ny: int, nz: int, lx: float = 0.0, ly: float = 0.0, lz: float = 0.0) -> str:
    """Frame::size_info: std::to_string of the counts and float origins."""
    return f"_{nx}_{ny}_{nz}_{lx:.6f}_{ly:.6f}_{lz:.6f}"


def write_traces(path_noext: str, tr: np.ndarray) -> str:
    """[n_recv][nt] traces in the reference's ascii layout."""
    tr = np.asarray(tr, dtype=np.float32)
    path = path_noext + ".txt"
    with open(path, "w") as f:
        for row in tr.reshape(tr.shape[0], -1):
            f.write("".join(f"{v:10.6e}\t" for v in row))
            f.write("\n")
    return path


def read_traces(path: str) -> np.ndarray:
    rows = []
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line:
                rows.append([float(t) for t in re.split(r"\s+", line)])
    return np.array(rows, dtype=np.float64)


def write_raw(path_noext: str, a: np.ndarray, nx: int, ny: int, nz: int) -> str:
    path = path_noext + size_info(nx, ny, nz) + ".raw"
    np.asarray(a, dtype=np.float32).tofile(path)
    return path
