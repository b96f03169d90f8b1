"""The jarvis-named drivers (tests/compat/*.cpp over jv/jarvis_compat.hpp)
and the sharded project job (jv_run_project_shard) on the GPU: the same
files and traces as jv_run_project and the in-memory calls."""
import subprocess
import threading

import numpy as np
import pytest

import make_golden as mg
from conftest import build_compat_driver, pkg, rel_l2

pytestmark = pytest.mark.gpu

jv = pkg()


def _read_outputs(project, d, s):
    out = {}
    for sh in range(s.shots.shape[0]):
        for c in ("vx", "vy", "vz"):
            out[f"{c}_{sh}"] = project.read_traces(f"{d}/out/{c}_seis_0_{sh}.txt")
    suf = project.size_info(s.nx, s.ny, s.nz)
    for nm in ("image_pp_0", "image_pp_laplace_0", "image_ps_0", "image_sp_0", "image_ss_0", "image_ipfd_0"):
        out[nm] = np.fromfile(f"{d}/out/{nm}{suf}.raw", np.float32)
    return out


def test_rtm_driver_matches_run_project(tmp_path, project):
    s = mg.case_survey("pin_w1")
    d1, d2 = str(tmp_path / "a") + "/", str(tmp_path / "b") + "/"
    project.write_project(d1, s)
    project.write_project(d2, s)
    exe = build_compat_driver("rtm_main", str(tmp_path))
    r = subprocess.run([exe, d1], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    with jv.Context.open(d2) as ctx:
        ctx.run_project()
    a, b = _read_outputs(project, d1, s), _read_outputs(project, d2, s)
    for k in b:
        assert np.array_equal(a[k], b[k]), k
    f = np.load(f"{mg.os.path.dirname(mg.__file__)}/ref_pin_w1.npz")
    assert rel_l2(a["image_pp_laplace_0"].reshape(s.nz, s.ny, s.nx), f["lap_pp"]) <= 5e-5


def test_forward_driver_matches_context(tmp_path, project, synth):
    s = synth.small_case(n=(16, 14, 12), pml=5, nt=50, seed=3)
    d = str(tmp_path / "p") + "/"
    project.write_project(d, s)
    exe = build_compat_driver("forward_main", str(tmp_path))
    out = str(tmp_path / "vz.raw")
    r = subprocess.run([exe, d, out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    with jv.Context.open(d) as ctx:
        vz = ctx.forward(0)[2]
    got = np.fromfile(out, np.float32).reshape(vz.shape)
    assert np.array_equal(got, vz)


def test_sharded_job_on_two_contexts_matches_single(tmp_path, project, synth):
    """Two ranks of one job, each its own context on the same GPU and its
    own host thread; the reduce callback sums through a host barrier (no
    kernel waits on another)."""
    s = synth.small_case(n=(18, 16, 14), pml=5, nt=60, seed=8,
                         shot_idx=[(4, 5, 2), (12, 9, 3), (9, 9, 9)])
    dref, dsh = str(tmp_path / "ref") + "/", str(tmp_path / "sh") + "/"
    project.write_project(dref, s)
    project.write_project(dsh, s)
    with jv.Context.open(dref) as ctx:
        ctx.run_project()

    world = 2
    slots = [None] * world
    bar = threading.Barrier(world, timeout=120)
    errors = []

    def make_reduce(rank):
        def reduce(arr):
            slots[rank] = arr.copy()
            bar.wait()
            total = slots[0] + slots[1]
            bar.wait()
            arr[:] = total
        return reduce

    ctxs = [jv.Context.open(dsh) for _ in range(world)]

    def run(rank):
        try:
            ctxs[rank].run_project_shard(rank, world, make_reduce(rank))
        except Exception as e:  # checked below
            errors.append(e)
            bar.abort()

    th = [threading.Thread(target=run, args=(r,)) for r in range(world)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    for c in ctxs:
        c.close()
    assert not errors, errors
    a, b = _read_outputs(project, dsh, s), _read_outputs(project, dref, s)
    for k in b:
        if k.startswith("v"):
            assert np.array_equal(a[k], b[k]), k
        else:
            assert rel_l2(a[k], b[k]) <= 1e-6, (k, rel_l2(a[k], b[k]))


def test_shard_arguments_checked(tmp_path, project, synth):
    s = synth.small_case(n=(10, 10, 10), pml=4, nt=10)
    d = str(tmp_path / "p") + "/"
    project.write_project(d, s)
    with jv.Context.open(d) as ctx:
        with pytest.raises(jv.JvError):
            ctx.run_project_shard(2, 2)
        with pytest.raises(jv.JvError):
            ctx.run_project_shard(0, 2)  # several ranks need a reduce function


def test_raw_model_project_matches_gms_project(tmp_path, project, synth):
    """model_path (GMS) and the raw-model keys (vp/vs/rho float32 files, x
    fastest, with their Frame) give the same job, bit for bit; with
    save_fld the images are also written as .fld files holding the same
    values under the reference Frame header."""
    s = synth.small_case(n=(18, 16, 14), pml=5, nt=60, seed=9, shot_idx=[(5, 6, 2), (11, 8, 3)])
    dg, dr = str(tmp_path / "gms") + "/", str(tmp_path / "raw") + "/"
    project.write_project(dg, s)
    project.write_project(dr, s, raw_model=True, save_fld=True)
    for d in (dg, dr):
        with jv.Context.open(d) as ctx:
            ctx.run_project()
    a, b = _read_outputs(project, dg, s), _read_outputs(project, dr, s)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    for nm in ("image_pp_0", "image_pp_laplace_0", "image_ps_0", "image_sp_0", "image_ss_0", "image_ipfd_0"):
        fr, img = project.read_fld(f"{dr}out/{nm}.fld")
        assert fr["type"] == 30 and (fr["n_rows"], fr["n_cols"], fr["n_slices"]) == (s.nx, s.ny, s.nz)
        assert fr["d"][0] == np.float32(s.dx) and fr["r"][2] == np.float32((s.nz - 1) * np.float32(s.dz))
        assert np.array_equal(img.reshape(-1), b[nm]), nm


def test_rtm_modules_driver_matches_run_project(tmp_path, project):
    """tests/compat/rtm_modules_main.cpp runs the job through the four module
    specialisations (pure_forward, rtm_forward with
    mpi_sub_forward_for_restruct, rtm_backward, rtm_reverse) and MigImage,
    with the reference's time-reverse loop of component calls, each a kernel
    launched on its own.  Its trace and image files equal jv_run_project's
    (graph-captured loops), bit for bit; its .fld of image_pp holds the
    same values."""
    s = mg.case_survey("pin_w1")
    d1, d2 = str(tmp_path / "a") + "/", str(tmp_path / "b") + "/"
    project.write_project(d1, s)
    project.write_project(d2, s)
    exe = build_compat_driver("rtm_modules_main", str(tmp_path))
    r = subprocess.run([exe, d1], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "geo_const: 4 2 1" in r.stdout
    with jv.Context.open(d2) as ctx:
        ctx.run_project()
    a, b = _read_outputs(project, d1, s), _read_outputs(project, d2, s)
    for k in b:
        assert np.array_equal(a[k], b[k]), k
    fr, img = project.read_fld(f"{d1}out/image_pp_0.fld")
    assert fr["type"] == 30 and np.array_equal(img.reshape(-1), b["image_pp_0"])


@pytest.mark.parametrize("w", [1, 3])
def test_reverse_ops_match_rtm_shot(synth, w):
    """The time-reverse loop driven one kernel at a time (jv_rtm_forward_pass,
    jv_rtm_reverse_begin, jv_rtm_reverse_op in the reference's order,
    jv_rtm_reverse_end) stacks the same images as jv_rtm_shot, bit for bit,
    with the same reconstruction check (its FP64 sums are atomic, so
    equal to rounding)."""
    import torch

    s = synth.small_case(n=(22, 18, 16), pml=6, nt=90, seed=21, rec_width=w)
    with jv.Context.from_survey(s) as ctx:
        obs = ctx.forward(0)
        ctx.image_reset()
        ctx.rtm_shot(0, obs)
        want = ctx.images()
        e_want = ctx.reconstruction_energy()
        i = ctx.info()
        dev = torch.from_numpy(np.stack(obs)).cuda()
        L = jv.lib()
        ctx.image_reset()
        assert L.jv_rtm_reverse_op(ctx._h, jv.OP_REVERSE_VEL, 0) == jv.JV_ESTATE  # no loop open
        assert L.jv_rtm_forward_pass(ctx._h, 0) == jv.JV_OK
        p = [dev[q].data_ptr() for q in range(3)]
        assert L.jv_rtm_reverse_begin(ctx._h, 0, p[0], p[1], p[2]) == jv.JV_OK
        for it in range(i.nt - 1, -1, -1):
            for op, t in ((jv.OP_INJECT_RECEIVERS, it), (jv.OP_REVERSE_VEL_PML, it), (jv.OP_BACKWARD_STRESS, it),
                          (jv.OP_INJECT_BOUNDARY_STRESS, it - 1), (jv.OP_REVERSE_VEL, it),
                          (jv.OP_BACKWARD_VEL_IMAGE, it), (jv.OP_INJECT_BOUNDARY_VEL, it - 1),
                          (jv.OP_REVERSE_STRESS_PML, it), (jv.OP_REVERSE_STRESS, it)):
                assert L.jv_rtm_reverse_op(ctx._h, op, t) == jv.JV_OK
        assert L.jv_rtm_reverse_end(ctx._h) == jv.JV_OK
        got = ctx.images()
        e_got = ctx.reconstruction_energy()
        assert L.jv_rtm_reverse_op(ctx._h, 99, 0) == jv.JV_ESTATE  # closed again
    for k in want:
        assert np.array_equal(got[k], want[k]), k
    for a, b in zip(e_got, e_want):
        assert abs(a - b) <= 1e-12 * abs(b), (e_got, e_want)
