"""The oracle against the reference itself.

tests/golden/ref_*.npz hold the outputs of the reference's own RTM driver
(oracle/build_ref.sh, run on a B200 by tests/golden/make_golden.py): the
traces it writes for every shot and its saved images.  The oracle, run on
the same regenerated inputs, must reproduce them:

* traces: relative L2 <= 5e-6 (the reference prints 7 significant digits
  and computes in FP32);
* uncompensated images (the reference saves I/Ip; multiplying back by its
  saved Ip recovers I): relative L2 <= 2e-5;
* Ip and the Laplacian of the uncompensated pp image: <= 5e-5;
* compensated images: <= 2e-3 -- dividing by the illumination amplifies
  the reference's own FP32 noise in dimly lit cells.
"""
import numpy as np
import pytest

import make_golden as mg
from conftest import rel_l2

CASES = list(mg.CASES)


def _problem(O, s):
    return O.Problem(s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.dt, s.fm, s.T, s.rec_width, s.shots, s.recvs,
                     s.vp, s.vs, s.rho)


@pytest.fixture(scope="module")
def runs(oracle):
    out = {}
    for name in CASES:
        s = mg.case_survey(name)
        p = _problem(oracle, s)
        traces, imgs = [], None
        for sh in range(s.shots.shape[0]):
            tr = oracle.forward(p, sh)
            traces.append(tr)
            imgs = oracle.rtm_shot(p, tr, sh, images=imgs)
        comp, lap = oracle.finalize_image(imgs, s.nx, s.ny, s.nz)
        out[name] = (s, traces, imgs, comp, lap)
    return out


@pytest.mark.parametrize("name", CASES)
def test_traces_match_reference(runs, name):
    s, traces, _, _, _ = runs[name]
    f = np.load(f"{mg.os.path.dirname(mg.__file__)}/ref_{name}.npz")
    for sh, tr in enumerate(traces):
        for c, t in zip(("vx", "vy", "vz"), tr):
            ref = f[f"tr_{c}_{sh}"]
            assert ref.shape == t.shape
            assert rel_l2(t, ref) <= 5e-6, (name, sh, c, rel_l2(t, ref))


@pytest.mark.parametrize("name", CASES)
def test_images_match_reference(runs, name):
    s, _, imgs, comp, lap = runs[name]
    f = np.load(f"{mg.os.path.dirname(mg.__file__)}/ref_{name}.npz")
    ip = f["img_ip"].astype(np.float64)
    assert rel_l2(imgs["ip"], ip) <= 5e-5
    assert rel_l2(lap["pp"], f["lap_pp"]) <= 5e-5
    for k in ("pp", "ps", "sp", "ss"):
        unc = f["img_" + k].astype(np.float64) * np.where(ip > 3.4e-38, ip, 1.0)
        assert rel_l2(imgs[k], unc) <= 2e-5, (name, k, rel_l2(imgs[k], unc))
        assert rel_l2(comp[k], f["img_" + k]) <= 2e-3, (name, k)


def test_fixture_layout():
    for name in CASES:
        f = np.load(f"{mg.os.path.dirname(mg.__file__)}/ref_{name}.npz")
        s = mg.case_survey(name)
        assert f["img_pp"].shape == (s.nz, s.ny, s.nx)
        assert f["tr_vx_0"].shape[1] == s.nt


@pytest.mark.parametrize("w", [1, 4])
def test_oracle_matches_reference_at_size(w):
    """cfg2 in full (200^3 + 20 CPML, 2000 steps, 40 000 receivers): the
    FP64 oracle's and the reference binary's outputs of the same shot, as
    make_size_pins.py stored them (16 receivers around the source; the raw
    images on the vertical plane through the source and on every 4th cell
    of the volume), agree within the reference's FP32 error; the
    whole-field figures of that run are in size_pins.json."""
    import json
    import os

    gold = os.path.dirname(mg.__file__)
    f = np.load(f"{gold}/size_cfg2_w{w}.npz")
    for c in ("vx", "vy", "vz"):
        assert rel_l2(f[f"oracle_tr_{c}"], f[f"ref_tr_{c}"]) <= 1e-4
    for k in ("ip", "pp", "ps", "sp", "ss"):
        # the vertical plane through the source holds the bright cells that set the whole-field norm
        assert rel_l2(f[f"oracle_{k}_y100"], f[f"ref_{k}_y100"]) <= 1e-4, k
        # the uniform sample of the volume misses them: there the FP32 noise of dim cells shows
        assert rel_l2(f[f"oracle_{k}_d4"], f[f"ref_{k}_d4"]) <= 5e-3, k
    with open(f"{gold}/size_pins.json") as fh:
        d = json.load(fh)[f"cfg2_w{w}"]
    assert d["grid_phy"] == [200, 200, 200] and d["nt"] == 2000 and d["n_recv"] == 40000
    for pair in ("gpu_vs_oracle", "gpu_vs_reference", "oracle_vs_reference"):
        assert max(d["traces"][pair].values()) <= 1e-5, pair
        assert max(d["raw_images"][pair].values()) <= 1e-4, pair
        assert d["laplacian_pp"][pair] <= 1e-4, pair


def test_boundary_store_precision_at_size():
    """cfg3 at half resolution (338 x 338 x 105 + 10 CPML, 1500 steps), the
    whole fields as make_size_pins.py measured them on a B200: with the FP32,
    FP16 and BF16 boundary stores the raw images stay within the workload's
    1e-3 bound against the FP64 oracle, and within 1e-4 of the FP32 store;
    the traces do not depend on the store."""
    import json
    import os

    with open(os.path.join(os.path.dirname(mg.__file__), "size_pins.json")) as fh:
        d = json.load(fh)["cfg3_half"]
    assert d["grid_phy"] == [338, 338, 105] and d["nt"] == 1500
    assert max(d["raw_images"]["gpu_vs_oracle"].values()) <= 1e-4
    assert max(d["raw_images"]["oracle_vs_reference"].values()) <= 1e-4
    for tag in ("fp16_store", "bf16_store"):
        p = d["boundary_store_precision"][tag]
        assert max(p["raw_images_vs_oracle"].values()) <= 1e-3, tag
        assert max(p["raw_images_vs_fp32_store"].values()) <= 1e-4, tag
        assert max(p["traces_vs_fp32_store"].values()) == 0.0, tag
