#!/usr/bin/env python
"""RTM throughput on B200: shots/h and Gcell-updates/s.

Workload (default): plain single-shot RTM on a 200^3 interior + 20 CPML
cells per face (240^3 gridext), d = 5 m, dt = 0.4 ms, 2000 steps, seeded
6-layer model with a Gaussian vp anomaly, source at cell (100,100,5),
200 x 200 receivers at z = 5, VOWR rec_width 1, FP32.  Synthetic seeded
inputs (no public data ship with the reference).

One step = one RTM shot: forward modelling with the VOWR boundary store,
then the time-reverse loop (source reconstruction, receiver
back-propagation, zero-lag imaging into FP64 stacks).  Observed traces are
modelled on the GPU once before timing.  Cell-updates per shot =
nt * (2 N_ext + N_phy).

  value  device-resident inputs; per-shot device time from CUDA events on
         the library's stream (jv_last_timing), max over ranks.
  e2e    the same shot through the host-pointer C ABI: H2D of the observed
         traces from pinned memory and D2H of the finalized images into
         pinned buffers reused per shot, inside the timed region (host clock
         around the synchronous calls).

--impl reference times the reference path's CPU implementation: the FP64
OpenMP restatement in oracle/ (the reference itself is GPU-only), on all
host cores, on a bounded sample of the same workload.

Multi-GPU (torchrun): shot replicas, one process per GPU, no collective
on the data path; value = shots of all ranks / max rank time.
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import re
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RTM shots/h & Gcell-updates/s, batched+served vs plain, 1 B200, rel-L2≤1e-3"


NOMINAL_HBM_GBS = 7700.0  # B200 HBM3e, NVIDIA's HGX figure; reported beside the measured peak


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(kernel: str):
    """dram bytes per launch of `kernel` from the committed ncu summary."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for fn in sorted(os.listdir(d)):
        if not fn.endswith((".md", ".txt")):
            continue
        with open(os.path.join(d, fn)) as f:
            for line in f:
                m = re.match(r"\s*traffic_bytes_per_launch\[(\w+)\]\s*[:=]\s*([0-9.eE+]+)", line)
                if m and m.group(1) == kernel:
                    return float(m.group(2))
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.p = None
        self.path = f"/tmp/jv_clocks_{os.getpid()}.csv"

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as f:
            for line in f:
                c = [x.strip() for x in line.split(",")]
                if len(c) < 9:
                    continue
                try:
                    sm.append(float(c[1]))
                    mx = max(mx, float(c[2]))
                except ValueError:
                    continue
                for n, v in zip(names, c[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def survey(args, synth):
    if args.grid:
        return synth.serving_grid(*args.grid, args.nt, seed=3)
    if args.n == 200 and args.nt == 2000:
        return synth.cfg2(rec_width=args.rec_width)
    return synth.scaled_cfg2(args.n, args.nt, rec_width=args.rec_width)


# algorithmic bytes per cell (FP32 fields, FP32 per-shot images): every array
# read once and written once per launch, neighbours reused on chip
BYTES_PER_CELL = {
    "vel_phy_bwd_image": 4 * (7 + 1 + 3 + 3 + 6) + 4 * 5 + 4 * 6 + 4 * 5,
    "vel_phy_rev": 4 * (7 + 1 + 6) + 4 * 6,
    "vel_phy_rtmfwd": 4 * (6 + 1 + 3) + 4 * 3,
    "vel_phy_fwd": 4 * (6 + 1 + 3) + 4 * 3,
    "stress_phy_bwd": 4 * (3 + 2 + 7) + 4 * 7,
    "stress_phy_rev": 4 * (3 + 2 + 7) + 4 * 7,
    "stress_phy_rtmfwd": 4 * (3 + 2 + 7) + 4 * 7,
    "stress_phy_fwd": 4 * (3 + 2 + 6) + 4 * 6,
}


# (arrays read, arrays written) per interior cell of each kernel: the
# footprint whose pointwise pass (jv_stream_probe) bounds what the kernel
# can move; the full-gridext kernels add CPML memory variables at the rim
FOOTPRINT = {
    "vel_phy_bwd_image": (25, 11), "vel_phy_rev": (14, 6), "vel_phy_rtmfwd": (10, 3), "vel_phy_fwd": (10, 3),
    "vel_fz_rtmfwd": (10, 3), "vel_fz_fwd": (10, 3),
    "stress_phy_bwd": (12, 7), "stress_phy_rev": (12, 7), "stress_phy_rtmfwd": (12, 7),
    "stress_fz_rev": (12, 7), "stress_fz_rtmfwd": (12, 7),
}


def attainable(jv, names, n, reps=5):
    """GB/s of the pointwise pass of each named kernel's footprint over n
    floats per array (arrays larger than L2): {footprint: GB/s}."""
    out = {}
    for k in names:
        fp = FOOTPRINT.get(k)
        if fp is not None and fp not in out:
            out[fp] = jv.stream_probe(fp[0], fp[1], n - n % 4, reps=reps)
    return out


def pml_bytes(s, name):
    """Algorithmic bytes of one CPML launch: per slab cell the fields, plus
    3 memory variables read+written per axis on which the cell absorbs."""
    m = s.pml
    NX, NY, NZ = s.nx + 2 * m, s.ny + 2 * m, s.nz + 2 * m

    def act(n):  # per-index: in the absorbing range of that axis
        a = np.zeros(n, bool)
        a[2:m] = True
        a[n - m:n - 2] = True
        return a

    ax, ay, az = act(NX), act(NY), act(NZ)
    ix = np.zeros(NX, bool); ix[2:NX - 2] = True
    iy = np.zeros(NY, bool); iy[2:NY - 2] = True
    iz = np.zeros(NZ, bool); iz[2:NZ - 2] = True
    px = np.zeros(NX, bool); px[m:NX - m] = True
    py = np.zeros(NY, bool); py[m:NY - m] = True
    pz = np.zeros(NZ, bool); pz[m:NZ - m] = True
    cells_all = ix.sum() * iy.sum() * iz.sum()
    cells = cells_all - px.sum() * py.sum() * pz.sum()
    # sum over PML cells of the number of absorbing axes: absorbing cells of
    # an axis are never physical, so count them over the inner box
    axes = ax[ix].sum() * iy.sum() * iz.sum() + ay[iy].sum() * ix.sum() * iz.sum() + az[iz].sum() * ix.sum() * iy.sum()
    if name == "vel_pml":
        per = 4 * (6 + 1 + 1 + 3) + 4 * 3
    elif name == "stress_pml":
        per = 4 * (3 + 3 + 6) + 4 * 6
    else:
        per = 4 * (3 + 3 + 7) + 4 * 7
    return float(cells * per + axes * 3 * 8)


# the full-gridext kernels (variant 4) do the work of two launches
FUSED = {"stress_fz_fwd": ("stress_phy_fwd", "stress_pml"),
         "stress_fz_rtmfwd": ("stress_phy_rtmfwd", "stress_pml_sau"),
         "stress_fz_rev": ("stress_phy_rev", "stress_pml_sau"),
         "vel_fz_fwd": ("vel_phy_fwd", "vel_pml"),
         "vel_fz_rtmfwd": ("vel_phy_rtmfwd", "vel_pml")}


def kernel_bytes(s, name):
    if name in BYTES_PER_CELL:
        return float(BYTES_PER_CELL[name] * s.n_phy)
    if name in ("vel_pml", "stress_pml", "stress_pml_sau"):
        return pml_bytes(s, name)
    if name in FUSED:
        return sum(kernel_bytes(s, k) for k in FUSED[name])
    return None


def cpu_sample(s, oracle, seconds_target=20.0, max_steps=200):
    """FP64 oracle on all host cores: a bounded sample of one RTM shot."""
    p = oracle.Problem(s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.dt, s.fm, s.T, s.rec_width, s.shots,
                       s.recvs, s.vp, s.vs, s.rho, nthreads=os.cpu_count() or 1)
    steps = 4
    t0 = time.perf_counter()
    cells = oracle.rtm_sample(p, steps)
    dt = time.perf_counter() - t0
    per_step = dt / steps
    steps2 = int(min(max_steps, max(4, seconds_target / max(per_step, 1e-6))))
    t0 = time.perf_counter()
    cells = oracle.rtm_sample(p, steps2)
    dt = time.perf_counter() - t0
    sec_per_shot = dt / steps2 * s.nt
    return {"shots_per_h": 3600.0 / sec_per_shot, "gcells": cells / dt / 1e9, "steps": steps2, "seconds": dt}


def _outputs(jv, plan):
    """Output arrays of every request, allocated and touched before timing
    (a serving loop reuses its buffers; first-touch page faults are the
    caller's allocator, not the server)."""
    outs = []
    for sv, k in plan:
        if k == jv.JOB_FORWARD:
            o = tuple(np.empty((sv.recvs.shape[0], sv.nt), np.float32) for _ in range(3))
        else:
            o = tuple(np.empty((sv.nz, sv.ny, sv.nx), np.float64) for _ in range(5))
        for a in o:
            a.fill(0)
        outs.append(o)
    return outs


def _served(jv, plan, outs, slots, timeout):
    """All requests submitted at once to a new server of `slots` slots;
    (seconds from the first submission to the last completion, stats)."""
    with jv.Server(slots=slots) as srv:
        t0 = time.perf_counter()
        subs = [srv.submit_survey(k, sv, outs=o) for (sv, k), o in zip(plan, outs)]
        for rid, _ in subs:
            if srv.wait(rid, timeout=timeout) != 0:
                raise RuntimeError("served request failed")
        dt = time.perf_counter() - t0
        st = srv.stats()
    return dt, st


def _repeat(jv, plan, outs, timeout, repeats):
    """1 slot and 4 slots, alternating, `repeats` times each; per config the
    median run (by time) and every run's requests/h."""
    runs = {1: [], 4: []}
    for _ in range(repeats):
        for slots in (1, 4):
            runs[slots].append(_served(jv, plan, outs, slots, timeout))
    med = {}
    for slots, rs in runs.items():
        rs = sorted(rs, key=lambda r: r[0])
        med[slots] = rs[len(rs) // 2]
    return runs, med


def serve_leg(jv, synth, n_req, repeats=3):
    """Heterogeneous requests through jv_server: grids of 48..112 cells per
    axis (+10 CPML), 400 steps, forward and RTM (the RTM requests model
    their own traces first), each with its own model and a full receiver
    plane; host buffers in and out, allocated before timing.  Served with 4
    slots against the same requests one at a time (1 slot), `repeats` runs
    of each, alternating, every run on a new server (its context pool
    starts empty); requests/h and p50/p99 latency from the server's own
    statistics (submission to completion) of the median run."""
    sizes = [48, 64, 80, 96, 112]
    surveys = {n: synth.scaled_cfg2(n, 400, pml=10, seed=30 + n) for n in sizes}
    plan = [(surveys[sizes[i % len(sizes)]], jv.JOB_RTM if i % 3 else jv.JOB_FORWARD) for i in range(n_req)]
    outs = _outputs(jv, plan)

    _served(jv, plan[:2], outs[:2], 2, 300.0)  # warm-up (module load, allocator pools), not counted
    runs, med = _repeat(jv, plan, outs, 600.0, repeats)
    (t1, st1), (t4, st4) = med[1], med[4]
    # forward: gridext; RTM: its own modelling, the forward pass and the
    # receiver propagation on gridext, the source reconstruction on gridphy
    cells = sum(sv.nt * (3 * sv.n_ext + sv.n_phy if k else sv.n_ext) for sv, k in plan)

    # a Poisson stream: requests arrive (seeded exponential gaps) while
    # others run, at half and at 0.9 of the 4-slot capacity just measured
    def poisson(rate, seed):
        rng = np.random.default_rng(seed)
        with jv.Server(slots=4) as srv:
            t0 = time.perf_counter()
            due = 0.0
            subs = []
            for (sv, k), o in zip(plan, outs):
                due += rng.exponential(1.0 / rate)
                pause = t0 + due - time.perf_counter()
                if pause > 0:
                    time.sleep(pause)
                subs.append(srv.submit_survey(k, sv, outs=o))
            for rid, _ in subs:
                if srv.wait(rid, timeout=600.0) != 0:
                    raise RuntimeError("served request failed")
            dt = time.perf_counter() - t0
            st = srv.stats()
        return {"offered_per_s": round(rate, 2), "achieved_per_s": round(n_req / dt, 2),
                "p50_ms": round(st["p50_ms"], 1), "p99_ms": round(st["p99_ms"], 1)}

    cap = n_req / t4
    stream = [poisson(f * cap, 40 + i) for i, f in enumerate((0.5, 0.9))]
    return {"requests": n_req, "unit": "requests/h",
            "poisson_4slots": stream,
            "mix": f"grids {sizes}^3 +10 CPML, nt 400, 2/3 RTM (own modelling first), 1/3 forward",
            "slots4": round(n_req / t4 * 3600.0, 1), "slots1": round(n_req / t1 * 3600.0, 1),
            "speedup": round(t1 / t4, 3),
            "runs": {"slots1": [round(n_req / t * 3600.0, 1) for t, _ in runs[1]],
                     "slots4": [round(n_req / t * 3600.0, 1) for t, _ in runs[4]]},
            "contexts_reused": {"slots1": st1["reused"], "slots4": st4["reused"]},
            "device_busy_slots1": round(st1["device_ms"] / (1000.0 * t1), 4),
            "p50_ms": {"slots4": round(st4["p50_ms"], 1), "slots1": round(st1["p50_ms"], 1)},
            "p99_ms": {"slots4": round(st4["p99_ms"], 1), "slots1": round(st1["p99_ms"], 1)},
            "gcell_updates_per_s": {"slots4": round(cells / t4 / 1e9, 2), "slots1": round(cells / t1 / 1e9, 2)},
            "note": f"median of {repeats} runs per slot count (alternating, each on a new server whose context pool "
                    "starts empty); latency counts from submission; all requests submitted at once; "
                    "poisson_4slots: seeded exponential arrival gaps at 0.5 and 0.9 of the slots4 rate; output "
                    "buffers allocated before timing; two warm-up requests on a server of their own are not counted"}


def serve_config_leg(jv, synth, n_req, nt, rate, seed=5, nt_max=None, forward_share=0.0):
    """Serving at the configured grid sizes: n_req requests on grids drawn
    (seeded) from {120^3, 200^3, 320^3, 480 x 480 x 200} + 20 CPML, seeded
    layered models and source positions, arriving as a Poisson stream at
    `rate` requests/s, served with 4 slots under the default HBM budget.
    Step counts: nt, or drawn uniformly from [nt, nt_max]; a share of
    forward_share of the requests is forward modelling, the others RTM
    (each modelling its own traces first)."""
    grids = [(120, 120, 120), (200, 200, 200), (320, 320, 320), (480, 480, 200)]
    rng = np.random.default_rng(seed)
    picks = [grids[int(k)] for k in rng.permutation(np.arange(n_req) % len(grids))]
    nts = [int(rng.integers(nt, nt_max + 1)) if nt_max else nt for _ in picks]
    kinds = [jv.JOB_FORWARD if rng.random() < forward_share else jv.JOB_RTM for _ in picks]
    reqs = [synth.serving_grid(*g, n, seed=300 + k) for k, (g, n) in enumerate(zip(picks, nts))]
    plan = list(zip(reqs, kinds))
    outs = _outputs(jv, plan)
    # forward: one pass; RTM: own modelling + forward pass + reverse loop
    cells = sum(r.nt * (r.n_ext if k == jv.JOB_FORWARD else 3 * r.n_ext + r.n_phy) for r, k in plan)
    with jv.Server(slots=4) as srv:
        t0 = time.perf_counter()
        due, subs = 0.0, []
        for (r, k), o in zip(plan, outs):
            due += rng.exponential(1.0 / rate)
            pause = t0 + due - time.perf_counter()
            if pause > 0:
                time.sleep(pause)
            subs.append(srv.submit_survey(k, r, outs=o))
        for rid, _ in subs:
            if srv.wait(rid, timeout=1800.0) != 0:
                raise RuntimeError("served request failed")
        dt = time.perf_counter() - t0
        st = srv.stats()
    return {"requests": n_req, "grids": ["x".join(map(str, g)) for g in picks], "pml": 20,
            "nt": nts if nt_max else nt, "kinds": ["forward" if k == jv.JOB_FORWARD else "rtm" for _, k in plan],
            "offered_per_s": rate, "unit": "requests/h", "value": round(n_req / dt * 3600.0, 1),
            "gcell_updates_per_s": round(cells / dt / 1e9, 2), "p50_ms": round(st["p50_ms"], 1),
            "p99_ms": round(st["p99_ms"], 1), "seconds": round(dt, 2), "contexts_reused": st["reused"],
            "note": "4 slots; RTM requests model their own traces, then migrate; latency from submission"}


def serve_sweep(jv, synth, n_req, rates):
    """The serving configuration as specified, opt-in (--serve-sweep): a
    Poisson stream at each rate, nt drawn from 1500-3000, half forward
    modelling and half RTM, grids from the configured four."""
    return [serve_config_leg(jv, synth, n_req, 1500, r, seed=50 + i, nt_max=3000, forward_share=0.5)
            for i, r in enumerate(rates)]


def batched_leg(jv, synth, torch, device, n_shots, nt, n_models, nt_mixed, repeats=3):
    """The batched configuration, bounded in shots and steps.

    (a) n_shots shots at seeded surface positions (depth 5 cells) on one
    160^3 + 16 CPML model, nt steps: one jv_rtm_batch of all shots and one
    finalize, against one jv_rtm_shot + finalize per shot.  The context
    makes the measured kernel choice (kernel_variant -1: variant and run
    chunking) when it is created.  Traces are modelled first (not timed);
    host traces in, host images out.
    (b) n_models independent seeded models with interior sizes drawn
    uniformly from {80, 96, 120, 160, 200}^3 (+16 CPML), nt_mixed steps, one
    RTM request each (modelling its own traces) through jv_server with 4
    slots, against the same requests one at a time (1 slot), `repeats` runs
    of each."""
    import dataclasses
    rng = np.random.default_rng(64)
    base = synth.scaled_cfg2(160, nt, pml=16, seed=64)
    pos = np.stack([rng.integers(8, 152, n_shots), rng.integers(8, 152, n_shots), np.full(n_shots, 5)], axis=1)
    s = dataclasses.replace(base, shots=(pos * 5.0).astype(np.float32), name="shots_160")
    out = {}
    with jv.Context.from_survey(s, device=device, kernel_variant=-1) as ctx:
        i = ctx.info()
        kcfg = ctx.kernel_config()
        obs = [ctx.forward(k) for k in range(n_shots)]
        himg = torch.empty((8, s.nz, s.ny, s.nx), dtype=torch.float32, pin_memory=True)
        hout = [himg[q].numpy() for q in range(8)]
        ctx.rtm_shot(0, obs[0])  # warm-up: graph capture
        ctx.finalize(out=hout)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for k in range(n_shots):
            ctx.rtm_shot(k, obs[k])
            ctx.finalize(out=hout)
        torch.cuda.synchronize()
        tp = time.perf_counter() - t0
        t0 = time.perf_counter()
        ctx.rtm_batch(list(range(n_shots)), obs)
        ctx.finalize(out=hout)
        torch.cuda.synchronize()
        tb = time.perf_counter() - t0
        cells = nt * (2 * i.n_ext + i.n_phy)
        out["shots_one_model"] = {
            "grid_phy": [160, 160, 160], "pml": 16, "nt": nt, "shots": n_shots, "n_recv": i.n_recv,
            "kernel_choice": {"kernel_variant": kcfg["kernel_variant"], "run_chunks": kcfg["run_chunks"]},
            "unit": "shots/h", "plain": round(n_shots / tp * 3600.0, 1), "batched": round(n_shots / tb * 3600.0, 1),
            "gcell_updates_per_s": {"plain": round(n_shots * cells / tp / 1e9, 2),
                                    "batched": round(n_shots * cells / tb / 1e9, 2)}}
        del obs

    sizes = [int(n) for n in rng.choice([80, 96, 120, 160, 200], n_models)]
    models = [synth.scaled_cfg2(n, nt_mixed, pml=16, seed=200 + k) for k, n in enumerate(sizes)]
    # own modelling (gridext), the RTM forward pass (gridext), the reverse
    # loop's receiver (gridext) and source (gridphy) propagations: the
    # count of the single-shot and serving figures
    cells = sum(nt_mixed * (3 * m.n_ext + m.n_phy) for m in models)

    plan = [(m, jv.JOB_RTM) for m in models]
    outs = _outputs(jv, plan)
    warm = {}
    for (m, k), o in zip(plan, outs):
        warm.setdefault(m.nx, ((m, k), o))
    _served(jv, [w[0] for w in warm.values()], [w[1] for w in warm.values()], 2, 900.0)  # warm-up, not counted
    runs, med = _repeat(jv, plan, outs, 900.0, repeats)
    (t1, st1), (t4, st4) = med[1], med[4]
    out["mixed_models"] = {
        "models": n_models, "sizes": {str(n): sizes.count(n) for n in sorted(set(sizes))}, "pml": 16,
        "nt": nt_mixed, "unit": "RTM shots/h", "slots1": round(n_models / t1 * 3600.0, 1),
        "slots4": round(n_models / t4 * 3600.0, 1), "speedup": round(t1 / t4, 3),
        "runs": {"slots1": [round(n_models / t * 3600.0, 1) for t, _ in runs[1]],
                 "slots4": [round(n_models / t * 3600.0, 1) for t, _ in runs[4]]},
        "contexts_reused": {"slots1": st1["reused"], "slots4": st4["reused"]},
        "gcell_updates_per_s": {"slots1": round(cells / t1 / 1e9, 2), "slots4": round(cells / t4 / 1e9, 2)},
        # the requests' propagation kernels' device time against the wall
        # time of the one-slot run: what a launch over several models could
        # still fill is the rest
        "device_busy_slots1": round(st1["device_ms"] / (1000.0 * t1), 4),
        "p50_ms": {"slots1": round(st1["p50_ms"], 1), "slots4": round(st4["p50_ms"], 1)},
        "p99_ms": {"slots1": round(st1["p99_ms"], 1), "slots4": round(st4["p99_ms"], 1)},
        "note": f"median of {repeats} runs per slot count (alternating, each on a new server whose context pool "
                "starts empty); each request models its own traces, then migrates; all submitted at once; latency "
                "from submission; output buffers allocated before timing; one warm-up request of each size on a "
                "server of its own is not counted; the configured 48 models run "
                f"{nt_mixed} steps each"}
    return out


def extra_configs(jv, synth, torch, device):
    """The other configurations, one short measurement each (not the
    headline): cfg1 plain forward modelling in full, cfg2's RTM shot at
    rec_width 4 in full (with its accuracy against the size fixtures), and
    the large cfg3 grid's RTM shot with the FP16 boundary store, cut to a
    few time steps, with the measured kernel choice (kernel_variant -1, made
    when the context is created)."""
    out = {}
    s = synth.cfg1()
    with jv.Context.from_survey(s, device=device) as ctx:
        i = ctx.info()
        tr = torch.empty((3, max(i.n_recv, 1), i.nt), dtype=torch.float32, device=f"cuda:{device}")
        ptrs = [tr[q].data_ptr() for q in range(3)]
        ctx.forward_device(0, ptrs)  # warm-up (graph capture)
        ms = []
        for _ in range(3):
            ctx.forward_device(0, ptrs)
            ms.append(ctx.last_ms())
        t = min(ms) / 1000.0
        out["cfg1_forward"] = {"grid_phy": [s.nx, s.ny, s.nz], "pml": s.pml, "nt": s.nt, "n_recv": i.n_recv,
                               "ms_per_shot": round(1000 * t, 2), "shots_per_h": round(3600.0 / t, 1),
                               "gcell_updates_per_s": round(i.n_ext * s.nt / t / 1e9, 2)}
    # cfg2 at rec_width 4: the VOWR store keeps 4 layers per face (47 GB
    # of HBM in FP32), and the reconstruction is exact
    s = synth.cfg2(rec_width=4)
    with jv.Context.from_survey(s, device=device) as ctx:
        i = ctx.info()
        tr = torch.empty((3, i.n_recv, i.nt), dtype=torch.float32, device=f"cuda:{device}")
        ptrs = [tr[q].data_ptr() for q in range(3)]
        ctx.forward_device(0, ptrs)
        ctx.rtm_shot_device(0, ptrs)  # warm-up (graph capture, store allocation)
        ms = []
        for _ in range(2):
            ctx.rtm_shot_device(0, ptrs)
            ms.append(ctx.last_ms())
        t = min(ms) / 1000.0
        e0, e1 = ctx.reconstruction_energy()
        acc = accuracy_leg(ctx, s, tr, ptrs, 4)
        out["cfg2_rtm_w4"] = {
            "grid_phy": [s.nx, s.ny, s.nz], "pml": s.pml, "nt": s.nt, "rec_width": 4, "n_recv": i.n_recv,
            "shots_per_h": round(3600.0 / t, 1), "ms_per_shot": round(1000 * t, 1),
            "gcell_updates_per_s": round(s.nt * (2 * i.n_ext + i.n_phy) / t / 1e9, 2),
            "store_bytes": int(i.store_bytes_per_step) * (s.nt - 1), "store_on_device": bool(i.store_on_device),
            "reconstruction_residual_ratio": e1 / e0 if e0 > 0 else None, "accuracy": acc,
            "note": "best of 2 shots after one warm-up shot"}
        del tr
    nt3 = 40
    s = synth.cfg3(nt=nt3)
    with jv.Context.from_survey(s, device=device, precision=jv.JV_FP16, kernel_variant=-1) as ctx:
        i = ctx.info()
        kcfg = ctx.kernel_config()
        tr = torch.empty((3, i.n_recv, i.nt), dtype=torch.float32, device=f"cuda:{device}")
        ptrs = [tr[q].data_ptr() for q in range(3)]
        ctx.forward_device(0, ptrs)
        ctx.rtm_shot_device(0, ptrs)  # warm-up
        ctx.rtm_shot_device(0, ptrs)
        t = ctx.last_ms() / 1000.0
        cells = nt3 * (2 * i.n_ext + i.n_phy)
        out["cfg3_rtm_fp16_store"] = {
            "grid_phy": [s.nx, s.ny, s.nz], "pml": s.pml, "nt_run": nt3, "nt_config": 3000, "n_recv": i.n_recv,
            "ms_per_step": round(1000 * t / nt3, 3), "gcell_updates_per_s": round(cells / t / 1e9, 2),
            "shot_s_at_3000_steps": round(t / nt3 * 3000, 1),
            "store_bytes_per_step": int(i.store_bytes_per_step), "device_bytes": int(i.device_bytes),
            "kernel_choice": {k: kcfg[k] for k in ("kernel_variant", "run_chunks", "tile_gx", "pml_min_blocks")},
            "note": "the configured 3000 steps cut to 40 to keep the bench short; per-step cost is constant"}
        del tr
    return out


SIZE_FIXTURES = {("cfg2_rtm_200_w1", 1): "size_cfg2_w1", ("cfg2_rtm_200_w4", 4): "size_cfg2_w4"}


def accuracy_leg(ctx, s, obs, ptrs, rec_width):
    """The timed configuration's accuracy, measured on this run: one RTM
    shot's traces of 16 receivers around the source and its five raw images
    on the vertical plane y = 100 through the source and on every 4th cell
    of every axis, against the FP64 oracle's and the reference binary's
    outputs of the same shot (tests/golden/size_cfg2_w*.npz, made by
    tests/golden/make_size_pins.py on a B200), with the reference's own
    error on each sample beside them; plus the whole-field figures that
    script measured (tests/golden/size_pins.json)."""
    name = SIZE_FIXTURES.get((s.name, rec_width))
    gold = os.path.join(ROOT, "tests", "golden")
    path = os.path.join(gold, f"{name}.npz") if name else None
    if not path or not os.path.exists(path):
        return {"unavailable": f"no size fixture for {s.name} at rec_width {rec_width}"}
    f = np.load(path)
    sub = f["subset"]
    ctx.image_reset()
    ctx.rtm_shot_device(0, ptrs)
    img = ctx.images()
    ctx.image_reset()

    def rl2(a, b):
        a = np.asarray(a, np.float64)
        b = np.asarray(b, np.float64)
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    import torch
    samples = {"plane_y100": ("y100", lambda a: a[:, 100]), "volume_every_4th": ("d4", lambda a: a[2::4, 2::4, 2::4])}
    idx = torch.as_tensor(np.asarray(sub, dtype=np.int64), device=obs.device)
    tr = [obs[q].index_select(0, idx).cpu().numpy() for q in range(3)]
    comps = ("vx", "vy", "vz")
    out = {"traces_16_receivers": {
        "vs_fp64_oracle": max(rl2(tr[q], f[f"oracle_tr_{c}"]) for q, c in enumerate(comps)),
        "vs_reference_binary": max(rl2(tr[q], f[f"ref_tr_{c}"]) for q, c in enumerate(comps)),
        "reference_binary_vs_fp64_oracle": max(rl2(f[f"ref_tr_{c}"], f[f"oracle_tr_{c}"]) for c in comps)}}
    for label, (sk, cut) in samples.items():
        out[label] = {}
        for k in ("ip", "pp", "ps", "sp", "ss"):
            a = cut(img[k])
            out[label][k] = {"vs_fp64_oracle": rl2(a, f[f"oracle_{k}_{sk}"]),
                             "vs_reference_binary": rl2(a, f[f"ref_{k}_{sk}"]),
                             "reference_binary_vs_fp64_oracle": rl2(f[f"ref_{k}_{sk}"], f[f"oracle_{k}_{sk}"])}
    plane_worst = max(v["vs_fp64_oracle"] for v in out["plane_y100"].values())
    res = {"metric": "relative L2", **out, "image_bound_vs_fp64": 1e-3, "within_bound": plane_worst <= 1e-3,
           "sample": "this run's RTM shot: traces of 16 receivers around the source x all steps; the five raw "
                     "(stacked, uncompensated) images on the vertical plane y = 100 through the source (40 000 "
                     "cells, with the bright near-source cells that set the whole-field norm) and on every 4th "
                     "cell of every axis (125 000 cells of the dim volume, where FP32 noise shows for the "
                     "reference's own run too); within_bound: the plane, against FP64"}
    summ = os.path.join(gold, "size_pins.json")
    key = name[len("size_"):]
    if os.path.exists(summ):
        with open(summ) as fh:
            d = json.load(fh).get(key)
        if d:
            res["full_field"] = {"traces": d["traces"], "raw_images": d["raw_images"],
                                 "laplacian_pp": d["laplacian_pp"], "compensated": d["compensated"],
                                 "source": "tests/golden/size_pins.json (tests/golden/make_size_pins.py --run on "
                                           "one B200: every trace sample and every gridphy cell)"}
    return res


def spawn_ranks(args) -> int:
    """`--gpus N` (N > 1) without a launcher: start N ranks of this same
    command under torch.distributed.run (one process per GPU, rendezvous on
    127.0.0.1), as the reference's run script starts its MPI ranks itself
    (build/jarvis/jarvis_2_run:5-12).  Rank 0 prints the line; the exit
    code is the launcher's."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def dry_run(args) -> int:
    """The rank plumbing alone, on CPU (gloo): every rank takes its shard of
    the job's steps * world shots (replicas.shard_shots) and rank 0 prints
    one line with the world size and every rank's shard.  Nothing is timed."""
    import datetime
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    rep = importlib.import_module("domain-decomposition-release_b200.replicas")
    if world > 1:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    mine = rep.shard_shots(args.steps * world, rank, world)
    shards = [None] * world
    if world > 1:
        dist.all_gather_object(shards, mine)
        dist.barrier()
        dist.destroy_process_group()
    else:
        shards = [mine]
    if rank == 0:
        print(json.dumps({"dry_run": True, "impl": args.impl, "n_gpus": world, "steps": args.steps,
                          "shots": args.steps * world, "shards": shards}), flush=True)
    return 0


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    synth = importlib.import_module("domain-decomposition-release_b200.synth")
    s = survey(args, synth)
    p = O.Problem(s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.dt, s.fm, s.T, s.rec_width, s.shots, s.recvs, s.vp,
                  s.vs, s.rho, nthreads=os.cpu_count() or 1)
    sample_steps = args.ref_sample_steps
    for _ in range(args.warmup):
        O.rtm_sample(p, max(2, sample_steps // 4))
    times, cells = [], 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cells = O.rtm_sample(p, sample_steps)
        times.append(time.perf_counter() - t0)
    tot = sum(times)
    sec_per_shot = tot / args.steps / sample_steps * s.nt
    value = 3600.0 / sec_per_shot
    sample = (f"{sample_steps} of {s.nt} time steps of each propagation of one RTM shot "
              f"({s.nx}^3 + {s.pml} CPML, {s.recvs.shape[0]} receivers), scaled to a full shot")
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "shots/h",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1000 * sec_per_shot, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "gcell_updates_per_s": round(cells * args.steps / tot / 1e9, 4),
        "config": {"workload": s.name, "grid_phy": [s.nx, s.ny, s.nz], "pml": s.pml, "nt": s.nt,
                   "rec_width": s.rec_width, "n_recv": int(s.recvs.shape[0]), "parallelism": "cpu-openmp"},
        "cpu_baseline": {"value": round(value, 4), "unit": "shots/h", "cores": os.cpu_count(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(value, 4), "unit": "shots/h", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="jv", choices=["jv", "reference"])
    ap.add_argument("--n", type=int, default=200, help="interior cells per axis")
    ap.add_argument("--grid", type=int, nargs=3, metavar=("NX", "NY", "NZ"), default=None,
                    help="a non-cubic interior instead of --n (seeded dipping layers, 5 m cells, 20 CPML)")
    ap.add_argument("--nt", type=int, default=2000)
    ap.add_argument("--rec-width", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-profile", action="store_true")
    ap.add_argument("--no-serve", action="store_true", help="skip the request-server leg")
    ap.add_argument("--serve-requests", type=int, default=24)
    ap.add_argument("--no-extra", action="store_true", help="skip the cfg1 / cfg3 side measurements")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-configuration leg")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the accuracy leg")
    ap.add_argument("--serve-config-requests", type=int, default=6,
                    help="requests of the configured-grid serving sample (0 skips it)")
    ap.add_argument("--serve-config-nt", type=int, default=1500)
    ap.add_argument("--serve-sweep", default="",
                    help="comma-separated arrival rates (requests/s) of the full serving sweep, e.g. 1,5,20,50 "
                         "(nt 1500-3000, half forward, half RTM); off by default")
    ap.add_argument("--serve-sweep-requests", type=int, default=8)
    ap.add_argument("--batch-shots", type=int, default=64, help="shots of the one-model batch (160^3)")
    ap.add_argument("--batch-nt", type=int, default=600, help="time steps of the one-model batch")
    ap.add_argument("--mixed-models", type=int, default=48, help="models of the mixed batch")
    ap.add_argument("--mixed-nt", type=int, default=200, help="time steps of each mixed-batch request")
    ap.add_argument("--ref-sample-steps", type=int, default=40)
    ap.add_argument("--variant", type=int, default=None, help="interior kernel variant (default: library default)")
    ap.add_argument("--store", default="fp32", choices=["fp32", "bf16", "fp16"],
                    help="boundary-store precision (wavefields are FP32 in every case)")
    ap.add_argument("--dry-run", action="store_true",
                    help="CPU only: start the ranks and print their shot shards, no GPU work")
    args = ap.parse_args()
    if args.warmup < 3:
        print("bench.py: --warmup must be >= 3", file=sys.stderr)
        return 2
    if args.gpus < 1:
        print("bench.py: --gpus must be >= 1", file=sys.stderr)
        return 2
    launched = os.environ.get("WORLD_SIZE")
    if launched is None and args.gpus > 1:
        return spawn_ranks(args)
    if launched is not None and int(launched) != args.gpus:
        print(f"bench.py: --gpus {args.gpus} but the launcher started WORLD_SIZE={launched} ranks", file=sys.stderr)
        return 2
    if args.dry_run:
        return dry_run(args)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)

    jv = importlib.import_module("domain-decomposition-release_b200")
    s = survey(args, jv.synth)
    kopts = {} if args.variant is None else {"kernel_variant": args.variant}
    if args.store != "fp32":
        kopts["precision"] = {"bf16": jv.JV_BF16, "fp16": jv.JV_FP16}[args.store]
    ctx = jv.Context.from_survey(s, device=local, **kopts)
    # the job: steps * world shots at the survey's source position, shot s
    # on rank s % world (replicas.shard_shots); per-shot work does not
    # depend on the position, so the per-rank work is fixed as N grows
    rep = importlib.import_module("domain-decomposition-release_b200.replicas")
    n_job = args.steps * world
    ctx.set_geometry(np.repeat(s.shots[:1], n_job, axis=0), s.recvs)
    mine = rep.shard_shots(n_job, rank, world)
    info = ctx.info()
    kcfg = ctx.kernel_config()  # the knobs the context's creation-time timing chose
    nrec, nt = info.n_recv, info.nt
    obs = torch.empty((3, nrec, nt), dtype=torch.float32, device=f"cuda:{local}")
    ptrs = [obs[i].data_ptr() for i in range(3)]
    ctx.forward_device(0, ptrs)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        ctx.image_reset()
        ctx.rtm_shot_device(0, ptrs)

    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    dev_ms = 0.0
    t0 = time.perf_counter()
    for shot in mine:
        ctx.rtm_shot_device(shot, ptrs)
        dev_ms += ctx.last_ms()
    barrier()
    wall = time.perf_counter() - t0
    clk = clocks.stop()

    dev_s = dev_ms / 1000.0
    if dist is not None:
        t = torch.tensor([dev_s], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_s = float(t.item())
    cells_per_shot = nt * (2 * info.n_ext + info.n_phy)
    shots = args.steps * world
    value = shots / dev_s * 3600.0
    gcells = shots * cells_per_shot / dev_s / 1e9

    # per-kernel device times (one instrumented shot, events on the library stream)
    roof = None
    prof = {}
    if not args.no_profile:
        ctx.set_profiling(True)
        ctx.rtm_shot_device(0, ptrs)
        prof = ctx.profile()
        ctx.set_profiling(False)
        tot = sum(v[0] for v in prof.values())
        name, (ms, n) = max(prof.items(), key=lambda kv: kv[1][0])
        b = kernel_bytes(s, name)
        peak, peak_kind = load_peaks()
        att = attainable(jv, prof.keys(), info.n_ext)
        if rank == 0:
            print(f"per-kernel device time, one instrumented RTM shot ({s.name}, CUDA events on the library stream):",
                  file=sys.stderr)
            print(f"  {'kernel':22s} {'launches':>8s} {'us/launch':>10s} {'share':>7s} {'alg. bytes':>12s} "
                  f"{'GB/s':>8s} {'of peak':>8s} {'of attainable':>14s}", file=sys.stderr)
            for k, (kms, kn) in sorted(prof.items(), key=lambda kv: -kv[1][0]):
                kb = kernel_bytes(s, k)
                us = 1000.0 * kms / max(kn, 1)
                gbs = kb / (us * 1e-6) / 1e9 if kb else float("nan")
                a = att.get(FOOTPRINT.get(k))
                print(f"  {k:22s} {kn:8d} {us:10.1f} {kms / tot:7.1%} {kb or 0:12.4g} {gbs:8.0f} "
                      f"{gbs / peak:8.1%} {(gbs / a) if a else float('nan'):14.1%}", file=sys.stderr)
            print("  attainable: " + ", ".join(f"{r} read + {w} written {g:.0f} GB/s" for (r, w), g in att.items()),
                  file=sys.stderr)
        if b is not None and n > 0:
            avg_s = ms / n / 1000.0
            ach = b / avg_s / 1e9
            tr = traffic_from_profiles(name)
            roof = {"bound": "hbm", "kernel": name, "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                    "frac": round(ach / peak, 4), "peak_source": peak_kind,
                    "peak_nominal": NOMINAL_HBM_GBS, "frac_nominal": round(ach / NOMINAL_HBM_GBS, 4),
                    "traffic": tr, "algorithmic_bytes_per_launch": b, "avg_launch_us": round(avg_s * 1e6, 2),
                    "share": round(ms / tot, 4) if tot > 0 else None}
            fp = FOOTPRINT.get(name)
            if fp in att:
                roof["attainable"] = {
                    "footprint": {"read": fp[0], "written": fp[1]}, "gbs": round(att[fp], 1),
                    "frac": round(ach / att[fp], 4),
                    "note": "jv_stream_probe: a pointwise float4 pass over the kernel's arrays (each "
                            f"{info.n_ext} floats, larger than L2), median of 5 launches; the bound of a pass "
                            "with that many arrays, which a two-array copy does not give"}

    accuracy = None
    if rank == 0 and not args.no_accuracy:
        accuracy = accuracy_leg(ctx, s, obs, ptrs, args.rec_width)

    # end to end through the host-pointer ABI: pinned H2D of the traces,
    # D2H of the 8 finalized images, every step
    e2e = None
    modes = None
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else args.steps
    if e2e_steps > 0:
        host = torch.empty((3, nrec, nt), dtype=torch.float32, pin_memory=True)
        host.copy_(obs.cpu())
        hobs = [host[i].numpy() for i in range(3)]
        # the eight finalized images land in pinned host buffers, reused per shot
        himg = torch.empty((8, s.nz, s.ny, s.nx), dtype=torch.float32, pin_memory=True)
        hout = [himg[q].numpy() for q in range(8)]
        # one untimed shot through the host path first: its first call sets up
        # the device trace buffer, the copy stream and the finalize buffer once
        # per context (about 0.3 s on cfg2), as the timed loop's warm-up does
        ctx.rtm_shot(0, hobs)
        ctx.finalize(out=hout)
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            ctx.rtm_shot(0, hobs)
            ctx.finalize(out=hout)
        barrier()
        te = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([te], dtype=torch.float64, device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            te = float(t.item())
        e2e = {"value": round(e2e_steps * world / te * 3600.0, 3), "unit": "shots/h",
               "h2d_bytes_per_step": int(3 * nrec * nt * 4), "d2h_bytes_per_step": int(8 * info.n_phy * 4)}

        # the same shots as one batch (jv_rtm_batch: the next shot's traces
        # copied while the current one runs, images read once per batch)
        # and as queued jobs (jv_submit / jv_wait), host buffers as above
        def timed(fn):
            barrier()
            t1 = time.perf_counter()
            fn()
            barrier()
            tt = time.perf_counter() - t1
            if dist is not None:
                tq = torch.tensor([tt], dtype=torch.float64, device=f"cuda:{local}")
                dist.all_reduce(tq, op=dist.ReduceOp.MAX)
                tt = float(tq.item())
            return round(e2e_steps * world / tt * 3600.0, 3)

        def batched():
            ctx.rtm_batch([0] * e2e_steps, [hobs] * e2e_steps)
            ctx.finalize(out=hout)

        def served():
            ids = [ctx.submit(jv.JOB_RTM, 0, obs=hobs) for _ in range(e2e_steps)]
            for i in ids:
                if ctx.wait(i) != 0:
                    raise RuntimeError("served job failed")
            ctx.finalize(out=hout)

        modes = {"unit": "shots/h", "plain_e2e": e2e["value"], "batched_e2e": timed(batched),
                 "served_e2e": timed(served),
                 "note": "plain: one jv_rtm_shot + jv_image_finalize per shot; batched: one jv_rtm_batch of the "
                         "shots, one finalize; served: the shots as queued RTM jobs, one finalize"}

    serving = None
    if world == 1 and not args.no_serve:
        serving = serve_leg(jv, jv.synth, args.serve_requests)
        if args.serve_config_requests > 0:
            serving["configured_grids"] = serve_config_leg(jv, jv.synth, args.serve_config_requests,
                                                           args.serve_config_nt, 1.0)
        if args.serve_sweep:
            serving["sweep"] = serve_sweep(jv, jv.synth, args.serve_sweep_requests,
                                           [float(r) for r in args.serve_sweep.split(",")])
    extra = None
    if world == 1 and not args.no_extra:
        extra = extra_configs(jv, jv.synth, torch, local)
    batched_cfg = None
    if world == 1 and not args.no_batched:
        batched_cfg = batched_leg(jv, jv.synth, torch, local, args.batch_shots, args.batch_nt, args.mixed_models,
                                  args.mixed_nt)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        c = cpu_sample(s, O)
        cpu = {"value": round(c["shots_per_h"], 4), "unit": "shots/h", "cores": os.cpu_count(), "kind": "port",
               "sample": f"FP64 oracle, {c['steps']} of {s.nt} time steps of each propagation of one shot, "
                         f"{c['seconds']:.1f} s, scaled to a full shot",
               "gcell_updates_per_s": round(c["gcells"], 4)}

    # the job's one exchange: sum the FP64 stacks of all replicas (after timing)
    reduce_ms = None
    if dist is not None:
        barrier()
        t0 = time.perf_counter()
        rep.reduce_images(ctx, device=local)
        barrier()
        reduce_ms = round(1000.0 * (time.perf_counter() - t0), 2)

    # kernels of one shot as the timed (graph) path launches them: the
    # instrumented shot advances the step counter every step, a captured
    # chunk of 32 steps once; plus the shot-end image stack
    launches = None
    if prof:
        chunks = 2 * (-(-nt // 32))
        launches = sum(v[1] for k, v in prof.items() if k != "step_advance") + chunks + 1
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "shots/h", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(1000 * dev_s / args.steps, 2), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "gcell_updates_per_s": round(gcells, 3),
        "config": {"workload": s.name, "grid_phy": [s.nx, s.ny, s.nz], "pml": s.pml, "nt": s.nt,
                   "rec_width": s.rec_width, "n_recv": nrec, "mode": "plain one-shot-per-call, graph time loop",
                   "job": f"{n_job} shots at the survey's source position, shot s on rank s % {world}",
                   "parallelism": f"shot replicas x{world}" if world > 1 else "single GPU",
                   "boundary_store": args.store,
                   "kernel_choice": {k: kcfg[k] for k in ("kernel_variant", "run_chunks", "tile_gx", "tile_gy",
                                                          "min_blocks", "planes_per_thread", "autotune")},
                   "l2": "inputs larger than L2 (each wavefield set > 700 MB)"},
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "accuracy": accuracy, "modes": modes, "serving": serving,
        "batched_config": batched_cfg,
        "other_configs": extra, "clocks": clk,
        "gpu_launches": launches * args.steps if launches else None,
        "gpu_launches_note": "kernels of the timed shots, counted from one instrumented shot (graph path)",
        "wall_s": round(wall, 3),
    }
    if reduce_ms is not None:
        line["image_allreduce_ms"] = reduce_ms
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
