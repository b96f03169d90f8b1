"""CUDA path (libjv.so, called through its C ABI) against the oracle and
against the reference's own outputs.

Tolerances (relative L2), FP32 GPU arithmetic:
  traces vs FP64 oracle ............................. 2e-5
  traces vs reference (7-digit text, FP32) .......... 5e-6
  raw stacked images / Ip vs FP64 oracle ............ 5e-5
  uncompensated images vs reference ................. 1e-5
  Ip vs reference ................................... 2e-5
  Laplacian of uncompensated pp vs reference ........ 1e-5
  compensated images (division by small Ip) ......... 2e-3
"""
import numpy as np
import pytest

import make_golden as mg
from conftest import pkg, rel_l2

pytestmark = pytest.mark.gpu

jv = pkg()


def _problem(O, s, w=None):
    return O.Problem(s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.dt, s.fm, s.T, w or s.rec_width, s.shots,
                     s.recvs, s.vp, s.vs, s.rho)


SMALL = [
    dict(n=(24, 20, 18), pml=6, nt=150, seed=3),
    dict(n=(17, 23, 13), pml=4, nt=120, seed=5, shot_idx=[(3, 20, 2)]),   # source near faces, pml at minimum
    dict(n=(40, 9, 11), pml=9, nt=100, seed=8, nrec=30),                  # random receivers anywhere
    dict(n=(8, 8, 8), pml=5, nt=60, seed=9, shot_idx=[(4, 4, 4)]),        # smallest allowed grid
]


# interior kernels: one plane per block, z-marching, x-vectorised, + TMA z-marching stress, + the stress update
# of the absorbing layers in the same TMA kernel (variant 4; even pml_num and nx, else variant 3's kernels)
VARIANTS = [0, 1, 2, 3, 4]


@pytest.mark.parametrize("kw", SMALL)
@pytest.mark.parametrize("graphs", [1, 0])
@pytest.mark.parametrize("variant", VARIANTS)
def test_forward_vs_oracle(oracle, synth, kw, graphs, variant):
    s = synth.small_case(**kw)
    ref = oracle.forward(_problem(oracle, s))
    with jv.Context.from_survey(s, use_graphs=graphs, graph_steps=7, kernel_variant=variant, zchunk=5) as ctx:
        tr = ctx.forward(0)
    assert tr[0].shape == ref[0].shape
    for a, b in zip(tr, ref):
        assert np.all(np.isfinite(a))
        assert rel_l2(a, b) <= 2e-5, rel_l2(a, b)


@pytest.mark.parametrize("name", list(mg.CASES))
def test_pins_vs_reference(synth, name):
    """Traces and images of the full reference job against the reference's
    own outputs (tests/golden/ref_*.npz).  Measured on the three cases:
    traces <= 1.2e-6, uncompensated images 2.1-7.5e-6, Laplacian of pp
    <= 6.5e-6, Ip <= 1.3e-5 relative L2.  The compensated images divide by
    a small illumination and amplify the reference's own FP32 noise (up to
    7.6e-4)."""
    s = mg.case_survey(name)
    f = np.load(f"{mg.os.path.dirname(mg.__file__)}/ref_{name}.npz")
    with jv.Context.from_survey(s) as ctx:
        ctx.image_reset()
        for sh in range(s.shots.shape[0]):
            tr = ctx.forward(sh)
            for c, t in zip(("vx", "vy", "vz"), tr):
                assert rel_l2(t, f[f"tr_{c}_{sh}"]) <= 5e-6, (sh, c, rel_l2(t, f[f"tr_{c}_{sh}"]))
            ctx.rtm_shot(sh, tr)
        raw = ctx.images()
        comp, lap = ctx.finalize()
    ip = f["img_ip"].astype(np.float64)
    assert rel_l2(raw["ip"], ip) <= 2e-5
    assert rel_l2(lap["pp"], f["lap_pp"]) <= 1e-5
    for k in ("pp", "ps", "sp", "ss"):
        unc = f["img_" + k].astype(np.float64) * np.where(ip > 3.4e-38, ip, 1.0)
        assert rel_l2(raw[k], unc) <= 1e-5, (k, rel_l2(raw[k], unc))
        assert rel_l2(comp[k], f["img_" + k]) <= 2e-3, (k, rel_l2(comp[k], f["img_" + k]))


@pytest.mark.parametrize("w", [1, 2, 3, 4])
@pytest.mark.parametrize("variant", VARIANTS)
def test_rtm_vs_oracle(oracle, synth, w, variant):
    s = synth.small_case(n=(22, 18, 21), pml=6, nt=140, seed=21, rec_width=w, anomaly=(0.1, 3.0),
                         shot_idx=[(11, 9, 3)])
    p = _problem(oracle, s, w)
    obs = oracle.forward(p)
    ref = oracle.rtm_shot(p, obs)
    obs32 = [o.astype(np.float32) for o in obs]
    with jv.Context.from_survey(s, kernel_variant=variant, zchunk=6) as ctx:
        ctx.rtm_shot(0, obs32)
        raw = ctx.images()
        comp, lap = ctx.finalize()
    for k in ("ip", "pp", "ps", "sp", "ss"):
        assert np.all(np.isfinite(raw[k]))
        assert rel_l2(raw[k], ref[k]) <= 5e-5, (w, k, rel_l2(raw[k], ref[k]))
    rc, rl = oracle.finalize_image(ref, s.nx, s.ny, s.nz)
    for k in ("pp", "ps", "sp", "ss"):
        assert rel_l2(lap[k], rl[k]) <= 5e-5
        assert rel_l2(comp[k], rc[k]) <= 2e-3


def test_images_stack_over_shots(synth):
    s = synth.small_case(n=(20, 16, 14), pml=5, nt=90, seed=4, shot_idx=[(5, 5, 2), (14, 10, 3)])
    with jv.Context.from_survey(s) as ctx:
        obs = [ctx.forward(i) for i in range(2)]
        singles = []
        for i in range(2):
            ctx.image_reset()
            ctx.rtm_shot(i, obs[i])
            singles.append(ctx.images())
        ctx.image_reset()
        for i in range(2):
            ctx.rtm_shot(i, obs[i])
        both = ctx.images()
    for k in both:
        assert rel_l2(both[k], singles[0][k] + singles[1][k]) <= 1e-12


def test_repeatable_and_graph_equivalent(synth):
    s = synth.small_case(n=(21, 19, 17), pml=6, nt=75, seed=12)
    outs = []
    for graphs, steps in ((1, 32), (1, 5), (0, 0)):
        with jv.Context.from_survey(s, use_graphs=graphs, graph_steps=steps) as ctx:
            a = ctx.forward(0)
            b = ctx.forward(0)
            ctx.rtm_shot(0, a)
            outs.append((a, b, ctx.image(jv.IMG_PP)))
    for a, b, im in outs:
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
        assert np.array_equal(im, outs[0][2])
        for x, y in zip(a, outs[0][0]):
            assert np.array_equal(x, y)


def test_project_roundtrip(tmp_path, synth, project):
    """jv_open + jv_run_project write the reference's files, readable with
    the reference's formats and equal to the in-memory results."""
    s = mg.case_survey("pin_w1")
    d = str(tmp_path / "proj")
    project.write_project(d, s)
    f = np.load(f"{mg.os.path.dirname(mg.__file__)}/ref_pin_w1.npz")
    with jv.Context.open(d + "/") as ctx:
        i = ctx.info()
        assert (i.grid.nx, i.grid.ny, i.grid.nz, i.nt, i.n_recv) == (s.nx, s.ny, s.nz, s.nt, s.recvs.shape[0])
        ctx.run_project()
    for sh in range(s.shots.shape[0]):
        for c in ("vx", "vy", "vz"):
            t = project.read_traces(f"{d}/out/{c}_seis_0_{sh}.txt")
            assert rel_l2(t, f[f"tr_{c}_{sh}"]) <= 1e-5
    suf = project.size_info(s.nx, s.ny, s.nz)
    pp = np.fromfile(f"{d}/out/image_pp_0{suf}.raw", np.float32).reshape(s.nz, s.ny, s.nx)
    lp = np.fromfile(f"{d}/out/image_pp_laplace_0{suf}.raw", np.float32).reshape(s.nz, s.ny, s.nx)
    assert rel_l2(pp, f["img_pp"]) <= 2e-3
    assert rel_l2(lp, f["lap_pp"]) <= 5e-5


def test_errors_are_status_codes(synth):
    s = synth.small_case(n=(12, 12, 12), pml=5, nt=20)
    with jv.Context.from_survey(s) as ctx:
        with pytest.raises(jv.JvError) as e:
            ctx.forward(5)
        assert e.value.code == jv.JV_EINVAL
        with pytest.raises(jv.JvError):
            ctx.image(9)
        ctx.set_geometry(np.array([[1e6, 0, 0]], np.float32), s.recvs)
        with pytest.raises(jv.JvError) as e:
            ctx.forward(0)
        assert "outside gridphy" in str(e.value)


OPTION_SETS = [
    dict(planes_per_thread=2),
    dict(pml_planes_per_thread=2),
    dict(min_blocks=3, pml_min_blocks=3),
    dict(tile_gx=3, tile_gy=7),
    dict(planes_per_thread=2, pml_planes_per_thread=2, tile_gx=5, tile_gy=9),
]


@pytest.mark.parametrize("kw", OPTION_SETS)
def test_launch_options_do_not_change_results(synth, kw):
    """Launch shapes, register budgets and planes per thread change only how
    the cells are assigned to threads (odd sizes, so partial groups, rows
    and plane pairs all occur).  A different register budget can change
    which multiply-adds the compiler contracts, so results agree to FP32
    rounding: traces 1e-6; images, whose correlation sums cancel, 2e-5
    (the tolerance against the FP64 oracle is 5e-5)."""
    s = synth.small_case(n=(23, 17, 15), pml=7, nt=70, seed=31, anomaly=(0.1, 3.0), shot_idx=[(11, 8, 3)])
    out = []
    for opts in (dict(), kw):
        with jv.Context.from_survey(s, **opts) as ctx:
            tr = ctx.forward(0)
            ctx.rtm_shot(0, tr)
            out.append((tr, ctx.images()))
    (t0, i0), (t1, i1) = out
    for a, b in zip(t0, t1):
        assert rel_l2(a, b) <= 1e-6
    for k in i0:
        assert rel_l2(i0[k], i1[k]) <= 2e-5, k


# grids on which variant 4's full-gridext stress and velocity kernels run (even pml_num and
# nx): region boundaries at every tile-row offset, the smallest pml, sources
# and receivers next to the absorbing layers
FULL = [
    dict(n=(26, 14, 16), pml=8, nt=120, seed=31, shot_idx=[(1, 2, 1)]),
    dict(n=(40, 12, 10), pml=10, nt=110, seed=32, nrec=40),
    dict(n=(12, 30, 22), pml=4, nt=130, seed=33, shot_idx=[(10, 27, 20)]),
    dict(n=(18, 9, 27), pml=6, nt=100, seed=34, shot_idx=[(9, 4, 13)]),
]


def _kernels(ctx):
    return set(ctx.profile())


@pytest.mark.parametrize("kw", FULL)
def test_full_stress_kernel_forward_vs_oracle(oracle, synth, kw):
    s = synth.small_case(**kw)
    ref = oracle.forward(_problem(oracle, s))
    with jv.Context.from_survey(s, kernel_variant=4) as ctx:
        tr = ctx.forward(0)
        ctx.set_profiling(True)
        ctx.forward(0)
        names = _kernels(ctx)
    assert {"stress_fz_fwd", "vel_fz_fwd"} <= names and not {"stress_pml", "vel_pml"} & names, names
    for a, b in zip(tr, ref):
        assert np.all(np.isfinite(a))
        assert rel_l2(a, b) <= 2e-5, rel_l2(a, b)


@pytest.mark.parametrize("kw", FULL[:2])
@pytest.mark.parametrize("w", [1, 4])
def test_full_stress_kernel_rtm_vs_oracle(oracle, synth, kw, w):
    s = synth.small_case(**dict(kw, rec_width=w))
    p = _problem(oracle, s, w)
    obs = oracle.forward(p)
    ref = oracle.rtm_shot(p, obs)
    obs32 = [o.astype(np.float32) for o in obs]
    with jv.Context.from_survey(s, kernel_variant=4) as ctx:
        ctx.set_profiling(True)
        ctx.rtm_shot(0, obs32)
        names = _kernels(ctx)
        raw = ctx.images()
    # the receiver side's velocity update keeps the split kernels
    assert {"stress_fz_rtmfwd", "stress_fz_rev", "vel_fz_rtmfwd", "vel_pml", "vel_phy_rev"} <= names, names
    assert "stress_pml_sau" not in names, names
    for k in ("ip", "pp", "ps", "sp", "ss"):
        assert np.all(np.isfinite(raw[k]))
        assert rel_l2(raw[k], ref[k]) <= 5e-5, (w, k, rel_l2(raw[k], ref[k]))


def test_full_stress_kernel_vs_oracle_at_size(oracle, synth):
    """Variant 4 against the oracle on a grid with several tiles per CTA and
    runs of planes that start inside a column, as accurate as variant 3's
    split kernels on the same problem."""
    s = synth.scaled_cfg2(44, 110, pml=10)
    p = _problem(oracle, s)
    obs = oracle.forward(p)
    ref = oracle.rtm_shot(p, obs)
    obs32 = [o.astype(np.float32) for o in obs]
    err = {}
    for v in (3, 4):
        with jv.Context.from_survey(s, kernel_variant=v) as ctx:
            tr = ctx.forward(0)
            ctx.rtm_shot(0, obs32)
            im = ctx.images()
        err[v] = ([rel_l2(a, b) for a, b in zip(tr, obs)], {k: rel_l2(im[k], ref[k]) for k in im})
    for e in err[4][0]:
        assert e <= 2e-5, err
    for k, e in err[4][1].items():
        assert e <= max(5e-5, 1.5 * err[3][1][k]), (k, err)


@pytest.mark.parametrize("prec,img_tol", [(jv.JV_FP16, 5e-5), (jv.JV_BF16, 1e-4)])
@pytest.mark.parametrize("w", [1, 4])
def test_16bit_boundary_store_vs_oracle(oracle, synth, prec, img_tol, w):
    """The VOWR boundary store in 16 bits with one FP32 scale per face box and
    step: the images against the FP64 oracle, next to the FP32 store's.
    Tolerances, relative L2: FP16 5e-5 and BF16 1e-4.  Measured on this case:
    0.9-1.2e-5 (FP16) and 1.4-1.9e-5 (BF16), against 0.7-1.0e-5 with the FP32
    store.  The replayed values only seed the rim of the reconstruction, so
    their 11 and 8 mantissa bits cost little."""
    s = synth.small_case(n=(22, 18, 21), pml=6, nt=140, seed=21, rec_width=w, anomaly=(0.1, 3.0),
                         shot_idx=[(11, 9, 3)])
    p = _problem(oracle, s, w)
    obs = oracle.forward(p)
    ref = oracle.rtm_shot(p, obs)
    obs32 = [o.astype(np.float32) for o in obs]
    err = {}
    for pr in (jv.JV_FP32, prec):
        with jv.Context.from_survey(s, precision=pr) as ctx:
            assert ctx.info().precision == pr
            ctx.rtm_shot(0, obs32)
            raw = ctx.images()
        err[pr] = {k: rel_l2(raw[k], ref[k]) for k in raw}
    print("image rel-L2 vs FP64 oracle, FP32 store:", err[jv.JV_FP32], "16-bit store:", err[prec])
    for k, e in err[prec].items():
        assert np.isfinite(e) and e <= img_tol, (k, err)


# grids wide enough that variant 4 cuts the x range into tiles (2-3 x tiles;
# the absorbing strips ride with the first and last tile)
WIDE = [
    dict(n=(260, 10, 12), pml=8, nt=90, seed=51, shot_idx=[(3, 5, 6)], nrec=30),
    dict(n=(300, 9, 10), pml=10, nt=80, seed=52, shot_idx=[(296, 4, 5)]),
    dict(n=(510, 8, 9), pml=4, nt=70, seed=53, shot_idx=[(255, 4, 4)], nrec=20),
]


@pytest.mark.parametrize("kw", WIDE)
def test_full_kernels_x_tiles_forward_vs_oracle(oracle, synth, kw):
    s = synth.small_case(**kw)
    ref = oracle.forward(_problem(oracle, s))
    with jv.Context.from_survey(s) as ctx:
        ctx.set_profiling(True)
        tr = ctx.forward(0)
        names = _kernels(ctx)
    # x-tiled grids: fused stress update, split velocity update
    assert {"stress_fz_fwd", "vel_pml", "vel_phy_fwd"} <= names and "vel_fz_fwd" not in names, names
    for a, b in zip(tr, ref):
        assert np.all(np.isfinite(a))
        assert rel_l2(a, b) <= 2e-5, rel_l2(a, b)


ZM3_WIDE = [
    dict(n=(400, 10, 9), pml=6, nt=60, seed=61),                                   # 2 tiles of 100 pairs
    dict(n=(484, 9, 10), pml=8, nt=60, seed=62, shot_idx=[(470, 4, 5)]),           # 2 tiles of 122 pairs
    dict(n=(676, 8, 8), pml=4, nt=50, seed=63, shot_idx=[(338, 4, 4)], nrec=20),   # 3 tiles of 114 pairs
]


@pytest.mark.parametrize("kw", ZM3_WIDE)
def test_zm3_x_tiles_vs_oracle(oracle, synth, kw):
    """Variant 3 on grids wider than one 248-cell row: its z-marching
    stress kernel cuts the rows into x tiles of at least 12 warps for every
    stress update, forward modelling, the RTM forward pass, the source
    reconstruction and the receiver side.  Traces and images against the
    oracle."""
    s = synth.small_case(**kw)
    p = _problem(oracle, s)
    obs = oracle.forward(p)
    ref = oracle.rtm_shot(p, obs)
    with jv.Context.from_survey(s, kernel_variant=3) as ctx:
        assert ctx.kernel_config()["kernel_variant"] == 3
        tr = ctx.forward(0)
        ctx.rtm_shot(0, [o.astype(np.float32) for o in obs])
        raw = ctx.images()
    for a, b in zip(tr, obs):
        assert rel_l2(a, b) <= 2e-5, rel_l2(a, b)
    for k in ("ip", "pp", "ps", "sp", "ss"):
        assert rel_l2(raw[k], ref[k]) <= 5e-5, (k, rel_l2(raw[k], ref[k]))


def test_full_kernels_x_tiles_rtm_vs_oracle(oracle, synth):
    s = synth.small_case(**dict(WIDE[0], rec_width=2, anomaly=(0.1, 3.0)))
    p = _problem(oracle, s, 2)
    obs = oracle.forward(p)
    ref = oracle.rtm_shot(p, obs)
    with jv.Context.from_survey(s) as ctx:
        ctx.set_profiling(True)
        ctx.rtm_shot(0, [o.astype(np.float32) for o in obs])
        names = _kernels(ctx)
        raw = ctx.images()
    assert {"stress_fz_rtmfwd", "stress_fz_rev"} <= names and "stress_pml_sau" not in names, names
    for k in ("ip", "pp", "ps", "sp", "ss"):
        assert rel_l2(raw[k], ref[k]) <= 5e-5, (k, rel_l2(raw[k], ref[k]))


@pytest.mark.parametrize("prec", [jv.JV_FP32, jv.JV_FP16])
def test_host_resident_boundary_store(synth, prec):
    """The boundary store in pinned host memory mapped into the device
    (store_mode JV_STORE_HOST, or a device budget too small under AUTO): the
    same images, bit for bit, as the store in HBM."""
    s = synth.small_case(n=(22, 18, 21), pml=6, nt=120, seed=21, rec_width=2, shot_idx=[(11, 9, 3)])
    out = {}
    for name, opts in (("device", dict(store_mode=jv.JV_STORE_DEVICE)), ("host", dict(store_mode=jv.JV_STORE_HOST)),
                       ("auto_small_budget", dict(store_mode=jv.JV_STORE_AUTO, store_budget=1))):
        with jv.Context.from_survey(s, precision=prec, **opts) as ctx:
            obs = ctx.forward(0)
            ctx.rtm_shot(0, obs)
            out[name] = (ctx.images(), ctx.info().store_on_device)
    assert out["device"][1] == 1 and out["host"][1] == 0 and out["auto_small_budget"][1] == 0
    for name in ("host", "auto_small_budget"):
        for k in out["device"][0]:
            assert np.array_equal(out[name][0][k], out["device"][0][k]), (name, k)


def test_measured_kernel_choice(oracle, synth):
    """kernel_variant -1: the context times the candidate variants on its
    grid at creation and keeps the fastest; the choice is reported, reused
    for the next context of the same shape, and its results match the
    oracle."""
    s = synth.small_case(n=(40, 24, 20), pml=8, nt=100, seed=61)
    ref = oracle.forward(_problem(oracle, s))
    picks = []
    for _ in range(2):
        with jv.Context.from_survey(s, kernel_variant=-1) as ctx:
            cfg = ctx.kernel_config()
            tr = ctx.forward(0)
        picks.append((cfg["kernel_variant"], cfg["pml_min_blocks"], cfg["run_chunks"]))
        assert cfg["kernel_variant"] in (2, 3, 4) and cfg["pml_min_blocks"] in (3, 4)
        assert (cfg["run_chunks"] > 0) == (cfg["kernel_variant"] == 4)
        # the float4 kernels' block shape: the default (0) or one more or one fewer block per row
        assert cfg["tile_gx"] in (0, 5, 10) and cfg["tile_gy"] == 0, (cfg["tile_gx"], cfg["tile_gy"])
        for a, b in zip(tr, ref):
            assert rel_l2(a, b) <= 2e-5, rel_l2(a, b)
    assert picks[0] == picks[1], picks  # the second context reuses the first one's choice
    with jv.Context.from_survey(s) as ctx:
        assert ctx.kernel_config()["kernel_variant"] == 4


def test_tile_with_a_mixed_warp(oracle, synth):
    """A grid whose x tiles fit one CTA only without rounding the physical
    pairs up to whole warps (484 cells, pml 6: two tiles of 121 pairs, 484 +
    8 threads): one warp then carries both the physical and the absorbing
    update.  Traces and images against the oracle."""
    s = synth.small_case(n=(484, 10, 9), pml=6, nt=50, seed=17, shot_idx=[(240, 5, 3)])
    p = _problem(oracle, s)
    obs = oracle.forward(p)
    ref = oracle.rtm_shot(p, obs)
    with jv.Context.from_survey(s) as ctx:
        assert ctx.kernel_config()["run_chunks"] > 0  # variant 4's kernels run
        tr = ctx.forward(0)
        ctx.rtm_shot(0, [o.astype(np.float32) for o in obs])
        raw = ctx.images()
    for a, b in zip(tr, obs):
        assert rel_l2(a, b) <= 2e-5, rel_l2(a, b)
    for k in ("ip", "pp", "ps", "sp", "ss"):
        assert rel_l2(raw[k], ref[k]) <= 5e-5, (k, rel_l2(raw[k], ref[k]))


@pytest.mark.parametrize("chunks", [1, 3, 7, 40])
def test_run_chunks_change_no_result(synth, chunks):
    """The run schedule of the persistent TMA kernels (run_chunks: chunks
    of each tile's planes) only decides which CTA updates which cells, so
    traces and images are bit-identical to the cost model's schedule; the
    chunking in use is reported (a count past the planes falls back to the
    cost model's)."""
    s = synth.small_case(n=(24, 20, 18), pml=6, nt=60, seed=3)
    out = {}
    for q in (0, chunks):
        with jv.Context.from_survey(s, run_chunks=q, autotune=0) as ctx:
            cfg = ctx.kernel_config()
            tr = ctx.forward(0)
            ctx.rtm_shot(0, tr)
            out[q] = (tr, ctx.images(), cfg["run_chunks"])
    nzi = s.nz + 2 * s.pml - 4
    assert out[chunks][2] == (chunks if chunks <= nzi else out[0][2]), (out[chunks][2], out[0][2])
    for a, b in zip(out[0][0], out[chunks][0]):
        assert np.array_equal(a, b)
    for k in out[0][1]:
        assert np.array_equal(out[0][1][k], out[chunks][1][k]), k


def test_default_autotune_is_result_neutral(synth):
    """By default a context times the knobs that cannot change a result
    (variant 4's run chunking among the cost model's best, the float4
    kernels' block shape) at creation: its traces and images equal those of
    a context with the cost model's fixed choice, bit for bit; the choice
    is reported and reused by the next context of the same shape."""
    s = synth.small_case(n=(40, 24, 20), pml=8, nt=80, seed=62)
    out, cfgs = {}, []
    for tune in (0, 1, 1):
        with jv.Context.from_survey(s, autotune=tune) as ctx:
            cfg = ctx.kernel_config()
            tr = ctx.forward(0)
            ctx.rtm_shot(0, tr)
            out[tune] = (tr, ctx.images())
        if tune:
            cfgs.append((cfg["run_chunks"], cfg["tile_gx"]))
        assert cfg["kernel_variant"] == 4 and cfg["run_chunks"] > 0 and cfg["autotune"] == tune
        assert cfg["tile_gx"] in (0, 5, 10) and cfg["tile_gy"] == 0
    assert cfgs[0] == cfgs[1], cfgs
    for a, b in zip(out[0][0], out[1][0]):
        assert np.array_equal(a, b)
    for k in out[0][1]:
        assert np.array_equal(out[0][1][k], out[1][1][k]), k


@pytest.mark.parametrize("variant", [4, 2])
def test_reconstruction_energy_check(synth, variant):
    """FP64 energy of the source wavefield at the end of the forward pass and
    after the reverse loop has reconstructed it to t = 0.  At rec_width 4
    the reconstruction is an exact time reversal (measured ratio 5e-11 on
    this case, FP32 rounding); below it is VOWR's approximation (6e-2 at
    width 1 on this small grid)."""
    ratio = {}
    for w in (1, 4):
        s = synth.small_case(n=(22, 18, 21), pml=6, nt=140, seed=21, rec_width=w, anomaly=(0.1, 3.0),
                             shot_idx=[(11, 9, 3)])
        with jv.Context.from_survey(s, kernel_variant=variant) as ctx:
            ctx.rtm_shot(0, ctx.forward(0))
            ef, er = ctx.reconstruction_energy()
        assert ef > 0 and np.isfinite(er)
        ratio[w] = er / ef
    assert ratio[4] < 1e-8, ratio
    assert 1e-3 < ratio[1] < 0.3, ratio
