"""Storage-precision study on the oracle: what FP16 or BF16 wavefield
storage (FP32 arithmetic, one power-of-two FP32 scale per z plane) costs in
trace and image error against the FP64 oracle.

TEST INFRASTRUCTURE: runs only the CPU oracle.  Usage (repository root):

    python oracle/store16_study.py [n] [nt ...]

n: interior cells per axis of a cfg2-style RTM problem (5 m spacing,
0.4 ms step, 10 CPML cells, full surface receiver plane); nt: step counts
(default 200 800).  Prints one line per (nt, storage): the largest trace
error over the three components and the relative L2 error of each raw
image (Ip, pp, ps, sp, ss).
"""
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))
import oracle as O  # noqa: E402

synth = importlib.import_module("domain-decomposition-release_b200.synth")


def rel_l2(a, b) -> float:
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def study(n: int, nt: int):
    s = synth.scaled_cfg2(n, nt, rec_width=1, pml=10)
    p = O.Problem(s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.dt, s.fm, s.T, 1, s.shots, s.recvs, s.vp, s.vs,
                  s.rho)
    obs = O.forward(p)
    ref = O.rtm_shot(p, obs)
    rows = []
    for kind in ("f32", "fp16", "bf16"):
        with O.store16(kind):
            tr = O.forward(p, precision="f32")
            img = O.rtm_shot(p, obs, precision="f32")
        rows.append((kind, max(rel_l2(a, b) for a, b in zip(tr, obs)),
                     {k: rel_l2(img[k], ref[k]) for k in ("ip", "pp", "ps", "sp", "ss")}))
    return rows


def main(argv):
    n = int(argv[1]) if len(argv) > 1 else 48
    nts = [int(a) for a in argv[2:]] or [200, 800]
    for nt in nts:
        for kind, et, ei in study(n, nt):
            print(f"n={n} nt={nt} storage={kind:5s} traces {et:.2e}  " +
                  "  ".join(f"{k} {v:.2e}" for k, v in ei.items()), flush=True)


if __name__ == "__main__":
    main(sys.argv)
