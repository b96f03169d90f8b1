"""Parity at the workload sizes: the GPU path, the FP64 oracle and the
reference's own binary on the full configurations.

The small pin cases (make_golden.py) tie the oracle to the reference; this
script measures the three against each other where the throughput is
quoted, on a GPU box:

  cfg1      plain forward modelling, 100^3 + 10 CPML, 1000 steps, 8 receivers
  cfg2_w1   single-shot RTM, 200^3 + 20 CPML, 2000 steps, 40 000 receivers,
            VOWR rec_width 1
  cfg2_w4   the same at rec_width 4 (the FP64 oracle's boundary store alone
            takes about 94 GB of host memory; skipped when the host has less)
  cfg3_half the precision configuration at half resolution (synth.cfg3_half:
            338 x 338 x 105 + 10 CPML, 20 m, 1500 steps): the GPU path with
            the FP32, FP16 and BF16 boundary stores

For each case, ``--run OUT`` writes the reference project, runs the
reference binary (oracle/_ref/jvref_rtm_w{1,4}, built by oracle/build_ref.sh),
runs the same shot through libjv and through the FP64 oracle on every host
core, and writes

  OUT/<case>.json        relative L2 errors over the whole fields (every
                         trace sample, every gridphy cell of the five raw
                         images, the Laplacian and the compensated images)
                         between each pair of the three, with run times;
  OUT/size_<case>.npz    a compact fixture for the GPU tests and the bench:
                         the FP64 oracle's and the reference's traces of 16
                         receivers around the source (cfg2) or of every
                         receiver (cfg1), and their raw images sampled at
                         every 4th cell of every axis and on the vertical
                         plane y = 100 through the source (cfg2).

``--collect OUT`` copies the fixtures and one summary (size_pins.json,
every case's figures) into tests/golden/.  Inputs are regenerated from
synth with fixed seeds, so the fixtures hold outputs only.

TEST INFRASTRUCTURE: the oracle and the reference binary are checkers; the
product never runs this file.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)
synth = importlib.import_module("domain-decomposition-release_b200.synth")
project = importlib.import_module("domain-decomposition-release_b200.project")

KINDS = ("ip", "pp", "ps", "sp", "ss")
# image samples: every 4th cell of every axis (a uniform sample of the whole
# volume) and the vertical plane y = 100 through the source
SAMPLES = ("d4", "y100")
# cfg2 receiver indices (j * 200 + i): 16 receivers around the source
SUBSET = [j * 200 + i for j in (85, 95, 105, 115) for i in (85, 95, 105, 115)]


def case_survey(name: str):
    if name == "cfg1":
        return synth.cfg1()
    if name == "cfg2_w1":
        return synth.cfg2(rec_width=1)
    if name == "cfg2_w4":
        return synth.cfg2(rec_width=4)
    if name == "cfg3_half":
        return synth.cfg3_half()
    raise KeyError(name)


def subset_of(name: str) -> list:
    """16 receivers around the source (indices into the survey's list)."""
    if name == "cfg3_half":  # a 169 x 169 receiver grid, the source under (84.5, 84.5)
        return [j * 169 + i for j in (76, 82, 88, 94) for i in (76, 82, 88, 94)]
    return SUBSET


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (d if d > 0 else 1.0))


def read_traces_fast(path: str, nrec: int, nt: int) -> np.ndarray:
    """The reference's ascii traces ([n_recv] lines of nt values)."""
    a = np.fromfile(path, dtype=np.float64, sep=" ")
    if a.size != nrec * nt:
        raise ValueError(f"{path}: {a.size} values, expected {nrec} x {nt}")
    return a.reshape(nrec, nt)


def sample(a: np.ndarray, key: str) -> np.ndarray:
    """An image sample of (nz, ny, nx) gridphy: 'd4' or 'y100'."""
    if key == "d4":
        return np.ascontiguousarray(a[2::4, 2::4, 2::4])
    return np.ascontiguousarray(a[:, 100, :])


def host_mem_gb() -> float:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) / 2**20
    except OSError:
        pass
    return 0.0


def run_reference(s, d: str) -> dict:
    project.write_project(d, s, rec_width_key=False)
    exe = os.path.join(ROOT, "oracle", "_ref", f"jvref_rtm_w{s.rec_width}")
    t0 = time.time()
    with open(os.path.join(d, "ref.log"), "w") as log:
        r = subprocess.run([exe, d + "/"], stdout=log, stderr=subprocess.STDOUT, timeout=3600)
    wall = time.time() - t0
    if r.returncode != 0:
        raise SystemExit(f"reference exit {r.returncode}")
    out = os.path.join(d, "out")
    nrec, nt = s.recvs.shape[0], s.nt
    tr = [read_traces_fast(os.path.join(out, f"{c}_seis_0_0.txt"), nrec, nt) for c in ("vx", "vy", "vz")]
    suf = project.size_info(s.nx, s.ny, s.nz)
    img = {}
    for key, fname in (("pp", "image_pp_0"), ("lap_pp", "image_pp_laplace_0"), ("ip", "image_ipfd_0"),
                       ("ps", "image_ps_0"), ("sp", "image_sp_0"), ("ss", "image_ss_0")):
        img[key] = np.fromfile(os.path.join(out, fname + suf + ".raw"), dtype=np.float32).reshape(s.nz, s.ny, s.nx)
    ip = img["ip"].astype(np.float64)
    comp = {k: img[k] for k in ("pp", "ps", "sp", "ss")}
    # the reference saves I / Ip (where Ip > 3.4e-38) and Ip: multiply back
    raw = {k: comp[k].astype(np.float64) * np.where(ip > 3.4e-38, ip, 1.0) for k in comp}
    raw["ip"] = ip
    with open(os.path.join(d, "ref.log")) as f:
        lines = f.read().splitlines()
    # the reference's own timers (cuda_toc lines) and the end of its log
    tail = "\n".join([ln for ln in lines if "time" in ln] + lines[-5:])[-4000:]
    return {"traces": tr, "raw": raw, "comp": comp, "lap_pp": img["lap_pp"], "wall_s": wall, "log_tail": tail}


def run_gpu(s, precision: int = 0) -> dict:
    jv = importlib.import_module("domain-decomposition-release_b200")
    with jv.Context.from_survey(s, precision=precision) as ctx:
        t0 = time.time()
        tr = ctx.forward(0)
        fwd_ms = ctx.last_ms()
        out = {"traces": [np.asarray(t) for t in tr], "forward_ms": fwd_ms}
        if not s.name.startswith("cfg1"):
            ctx.image_reset()
            ctx.rtm_shot(0, tr)
            out["rtm_ms"] = ctx.last_ms()
            out["raw"] = ctx.images()
            comp, lap = ctx.finalize()
            out["comp"], out["lap"] = comp, lap
            e0, e1 = ctx.reconstruction_energy()
            out["recon_energy_ratio"] = e1 / e0 if e0 > 0 else None
        out["wall_s"] = time.time() - t0
    return out


def run_oracle(s) -> dict:
    import oracle as O
    p = O.Problem(s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.dt, s.fm, s.T, s.rec_width, s.shots, s.recvs, s.vp,
                  s.vs, s.rho, nthreads=os.cpu_count() or 1)
    t0 = time.time()
    tr = O.forward(p)
    out = {"traces": list(tr), "forward_s": time.time() - t0}
    if not s.name.startswith("cfg1"):
        t1 = time.time()
        raw = O.rtm_shot(p, tr)
        out["rtm_s"] = time.time() - t1
        comp, lap = O.finalize_image(raw, s.nx, s.ny, s.nz)
        out["raw"], out["comp"], out["lap"] = raw, comp, lap
    out["cores"] = os.cpu_count()
    return out


def compare(s, g: dict, o: dict, r: dict) -> dict:
    res = {"traces": {}, "raw_images": {}, "laplacian_pp": {}, "compensated": {}}
    pairs = (("gpu_vs_oracle", g, o), ("gpu_vs_reference", g, r), ("oracle_vs_reference", o, r))
    for name, a, b in pairs:
        res["traces"][name] = {c: rel_l2(x, y) for c, x, y in zip(("vx", "vy", "vz"), a["traces"], b["traces"])}
    if "raw" in g:
        for name, a, b in pairs:
            res["raw_images"][name] = {k: rel_l2(a["raw"][k], b["raw"][k]) for k in KINDS}
            res["compensated"][name] = {k: rel_l2(a["comp"][k], b["comp"][k]) for k in ("pp", "ps", "sp", "ss")}
        lap_g, lap_o, lap_r = g["lap"]["pp"], o["lap"]["pp"], r["lap_pp"]
        res["laplacian_pp"] = {"gpu_vs_oracle": rel_l2(lap_g, lap_o), "gpu_vs_reference": rel_l2(lap_g, lap_r),
                               "oracle_vs_reference": rel_l2(lap_o, lap_r)}
        res["recon_energy_ratio_gpu"] = g.get("recon_energy_ratio")
    return res


def precision_study(g: dict, extra: dict, o: dict, r: dict) -> dict:
    """16-bit boundary stores (extra: "fp16" / "bf16" GPU runs) against the
    FP64 oracle, the reference and the FP32-store GPU run."""
    out = {}
    for tag, a in extra.items():
        out[tag] = {
            "raw_images_vs_oracle": {k: rel_l2(a["raw"][k], o["raw"][k]) for k in KINDS},
            "raw_images_vs_reference": {k: rel_l2(a["raw"][k], r["raw"][k]) for k in KINDS},
            "raw_images_vs_fp32_store": {k: rel_l2(a["raw"][k], g["raw"][k]) for k in KINDS},
            "laplacian_pp_vs_oracle": rel_l2(a["lap"]["pp"], o["lap"]["pp"]),
            "traces_vs_fp32_store": {c: rel_l2(x, y) for c, x, y in zip(("vx", "vy", "vz"), a["traces"], g["traces"])},
            "rtm_ms": round(a["rtm_ms"], 2)}
    return out


def fixture(name: str, s, o: dict, r: dict) -> dict:
    fx = {"case": np.array(name)}
    if name == "cfg1":
        for c, t in zip(("vx", "vy", "vz"), o["traces"]):
            fx[f"oracle_tr_{c}"] = t.astype(np.float32)
        for c, t in zip(("vx", "vy", "vz"), r["traces"]):
            fx[f"ref_tr_{c}"] = t.astype(np.float32)
        return fx
    sub = subset_of(name)
    fx["subset"] = np.array(sub, dtype=np.int32)
    for c, t in zip(("vx", "vy", "vz"), o["traces"]):
        fx[f"oracle_tr_{c}"] = t[sub].astype(np.float32)
    for c, t in zip(("vx", "vy", "vz"), r["traces"]):
        fx[f"ref_tr_{c}"] = t[sub].astype(np.float32)
    for pk in SAMPLES:
        for k in KINDS:
            fx[f"oracle_{k}_{pk}"] = sample(o["raw"][k], pk).astype(np.float32)
            fx[f"ref_{k}_{pk}"] = sample(r["raw"][k], pk).astype(np.float32)
    return fx


def run_case(name: str, out: str) -> None:
    s = case_survey(name)
    need = {"cfg2_w4": 150.0, "cfg2_w1": 40.0, "cfg3_half": 40.0}.get(name, 4.0)
    if host_mem_gb() < need:
        print(f"{name}: skipped, {host_mem_gb():.0f} GB of host memory available, {need:.0f} needed", flush=True)
        return
    d = tempfile.mkdtemp(prefix=f"jv_size_{name}_")  # the reference's trace files are large: kept out of OUT
    print(f"{name}: reference ...", flush=True)
    r = run_reference(s, d)
    print(f"{name}: reference {r['wall_s']:.1f} s; gpu ...", flush=True)
    g = run_gpu(s)
    extra = {}
    if name == "cfg3_half":
        extra = {"fp16_store": run_gpu(s, 2), "bf16_store": run_gpu(s, 1)}
    print(f"{name}: gpu {g['wall_s']:.1f} s; oracle ...", flush=True)
    o = run_oracle(s)
    print(f"{name}: oracle {o.get('forward_s', 0) + o.get('rtm_s', 0):.1f} s", flush=True)
    res = compare(s, g, o, r)
    if extra:
        res["boundary_store_precision"] = precision_study(g, extra, o, r)
    res.update({"case": name, "grid_phy": [s.nx, s.ny, s.nz], "pml": s.pml, "nt": s.nt, "rec_width": s.rec_width,
                "n_recv": int(s.recvs.shape[0]), "seed": s.seed,
                "times": {"reference_binary_wall_s": round(r["wall_s"], 2),
                          "gpu_forward_ms": round(g["forward_ms"], 2), "gpu_rtm_ms": round(g.get("rtm_ms", 0.0), 2),
                          "oracle_forward_s": round(o["forward_s"], 2), "oracle_rtm_s": round(o.get("rtm_s", 0.0), 2),
                          "oracle_cores": o["cores"]},
                "reference_log_tail": r["log_tail"]})
    with open(os.path.join(out, name + ".json"), "w") as f:
        json.dump(res, f, indent=1)
    np.savez_compressed(os.path.join(out, f"size_{name}.npz"), **fixture(name, s, o, r))
    shutil.rmtree(d, ignore_errors=True)
    print(json.dumps({k: res[k] for k in ("case", "traces", "raw_images", "laplacian_pp")}), flush=True)


def collect(out: str) -> None:
    """Adds the cases run into OUT to tests/golden/ (the fixtures, and their
    figures merged into size_pins.json)."""
    dst = os.path.join(HERE, "size_pins.json")
    summary = {}
    if os.path.exists(dst):
        with open(dst) as f:
            summary = json.load(f)
    for fn in sorted(os.listdir(out)):
        if fn.endswith(".json") and fn[:-5] in ("cfg1", "cfg2_w1", "cfg2_w4", "cfg3_half"):
            with open(os.path.join(out, fn)) as f:
                d = json.load(f)
            log = d.pop("reference_log_tail", "")
            d["reference_timers"] = [ln.strip() for ln in log.splitlines() if "time" in ln][:20]
            summary[fn[:-5]] = d
        if fn.startswith("size_") and fn.endswith(".npz"):
            shutil.copy(os.path.join(out, fn), os.path.join(HERE, fn))
            print("copied", fn)
    with open(dst, "w") as f:
        json.dump(summary, f, indent=1)
    print("wrote size_pins.json with", sorted(summary))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--run", metavar="OUT")
    ap.add_argument("--cases", nargs="+", default=["cfg1", "cfg2_w1"])
    ap.add_argument("--collect", metavar="OUT")
    a = ap.parse_args()
    if a.run:
        os.makedirs(a.run, exist_ok=True)
        for name in a.cases:
            run_case(name, a.run)
    if a.collect:
        collect(a.collect)


if __name__ == "__main__":
    main()
