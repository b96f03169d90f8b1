"""Generates the golden fixtures that pin the oracle to the reference.

The reference's own RTM driver is built by oracle/build_ref.sh into
oracle/_ref/jvref_rtm_w{1,4} (a CUDA program, so it runs on a GPU box).
This script

  --run-ref OUT   writes the pin projects (argfile.json, shot.txt,
                  rece.txt, model.gms) under OUT/<case>/ and runs the
                  matching reference binary in each (GPU box);
  --collect OUT   reads the reference outputs back and stores them, with the
                  case parameters, as tests/golden/ref_<case>.npz.

The inputs of every case are regenerated from synth.small_case() with the
fixed parameters below, so a fixture holds only the reference's outputs
plus the parameters needed to rebuild its inputs.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
synth = importlib.import_module("domain-decomposition-release_b200.synth")
project = importlib.import_module("domain-decomposition-release_b200.project")

# name -> small_case kwargs (+ rec_width selects the reference binary)
CASES = {
    "pin_w1": dict(n=(30, 26, 22), pml=8, nt=400, seed=11, rec_width=1, dx=10.0, dt=1e-3, fm=25.0,
                   shot_idx=[(15, 13, 3), (9, 17, 4)]),
    "pin_w4": dict(n=(30, 26, 22), pml=8, nt=400, seed=11, rec_width=4, dx=10.0, dt=1e-3, fm=25.0,
                   shot_idx=[(15, 13, 3), (9, 17, 4)]),
    "pin_anom_w1": dict(n=(28, 24, 26), pml=6, nt=300, seed=23, rec_width=1, dx=8.0, dt=8e-4, fm=30.0,
                        shot_idx=[(14, 12, 2)], anomaly=(0.15, 4.0)),
}


def case_survey(name: str):
    return synth.small_case(**CASES[name])


def run_ref(out: str) -> None:
    refdir = os.path.join(ROOT, "oracle", "_ref")
    for name in CASES:
        s = case_survey(name)
        d = os.path.join(out, name)
        project.write_project(d, s, rec_width_key=False)
        exe = os.path.join(refdir, f"jvref_rtm_w{s.rec_width}")
        with open(os.path.join(d, "ref.log"), "w") as log:
            r = subprocess.run([exe, d + "/"], stdout=log, stderr=subprocess.STDOUT, timeout=600)
        print(f"{name}: reference exit {r.returncode}")
        if r.returncode != 0:
            raise SystemExit(r.returncode)


def collect(out: str) -> None:
    for name in CASES:
        s = case_survey(name)
        d = os.path.join(out, name, "out")
        nshot = s.shots.shape[0]
        fx = {}
        for sh in range(nshot):
            for c in ("vx", "vy", "vz"):
                fx[f"tr_{c}_{sh}"] = project.read_traces(os.path.join(d, f"{c}_seis_0_{sh}.txt")).astype(np.float32)
        suf = project.size_info(s.nx, s.ny, s.nz)
        for key, fname in (("img_pp", "image_pp_0"), ("lap_pp", "image_pp_laplace_0"), ("img_ip", "image_ipfd_0"),
                           ("img_ps", "image_ps_0"), ("img_sp", "image_sp_0"), ("img_ss", "image_ss_0")):
            a = np.fromfile(os.path.join(d, fname + suf + ".raw"), dtype=np.float32)
            fx[key] = a.reshape(s.nz, s.ny, s.nx)
        fx["params"] = np.array(json.dumps(CASES[name]))
        dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"ref_{name}.npz")
        np.savez_compressed(dst, **fx)
        print("wrote", dst, os.path.getsize(dst), "bytes")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--run-ref", metavar="OUT")
    ap.add_argument("--collect", metavar="OUT")
    a = ap.parse_args()
    if a.run_ref:
        run_ref(a.run_ref)
    if a.collect:
        collect(a.collect)


if __name__ == "__main__":
    main()
