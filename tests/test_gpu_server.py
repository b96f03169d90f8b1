"""The request server (jv_server_*) on the GPU: requests of different grids,
models and kinds admitted into concurrent slots give the same traces and
images as each request run alone on a context of its own; the HBM budget
holds while they run; queued requests can be cancelled; the statistics
count what happened.  Every wait here is a host wait with a time limit."""
import dataclasses
import time

import numpy as np
import pytest

from conftest import pkg, rel_l2

pytestmark = pytest.mark.gpu

jv = pkg()
synth = pkg("synth")


def _cases():
    """Three problems of their own size, model and source."""
    return [synth.small_case(n=(18, 16, 14), pml=5, nt=80, seed=11, shot_idx=[(6, 7, 3)]),
            synth.small_case(n=(22, 20, 16), pml=6, nt=70, seed=12, shot_idx=[(11, 10, 2)], rec_width=2),
            synth.small_case(n=(20, 18, 24), pml=5, nt=90, seed=13, shot_idx=[(9, 9, 4)], nrec=25)]


def _alone(s, kind, obs=None, precision=jv.JV_FP32):
    with jv.Context.from_survey(s, precision=precision) as ctx:
        if kind == jv.JOB_FORWARD:
            return ctx.forward(0)
        if obs is None:
            obs = ctx.forward(0)
        ctx.image_reset()
        ctx.rtm_shot(0, obs)
        im = ctx.images()
        return tuple(im[k] for k in ("ip", "pp", "ps", "sp", "ss"))


def _check_same(kind, got, want):
    if kind == jv.JOB_FORWARD:
        for q in range(3):
            assert np.array_equal(got[q], want[q]), q
    else:
        for q in range(5):
            assert rel_l2(got[q], want[q]) <= 1e-12, q


def test_mixed_requests_match_each_run_alone():
    cases = _cases()
    plan = [(cases[0], jv.JOB_FORWARD, False), (cases[1], jv.JOB_RTM, True), (cases[2], jv.JOB_RTM, False),
            (cases[1], jv.JOB_FORWARD, False), (cases[0], jv.JOB_RTM, False), (cases[2], jv.JOB_FORWARD, False)]
    obs1 = _alone(cases[1], jv.JOB_FORWARD)
    want = [_alone(s, kind, obs1 if with_obs else None) for s, kind, with_obs in plan]
    with jv.Server(slots=4, budget=1 << 30) as srv:
        subs = [srv.submit_survey(kind, s, obs=obs1 if with_obs else None) for s, kind, with_obs in plan]
        for rid, _ in subs:
            assert srv.wait(rid, timeout=180.0) == jv.JV_OK
            assert srv.poll(rid) == (jv.JOB_DONE, jv.JV_OK)
        st = srv.stats()
    for (s, kind, _), (_, got), w in zip(plan, subs, want):
        _check_same(kind, got, w)
    assert st["submitted"] == 6 and st["completed"] == 6 and st["failed"] == 0
    assert st["running"] == 0 and st["queued"] == 0
    assert 0 < st["bytes_in_use"] <= st["budget"] and st["pooled"] >= 1  # idle contexts stay pooled
    assert 0 < st["p50_ms"] <= st["p99_ms"] and st["mean_ms"] > 0
    # each request's device time lies inside its submission-to-completion time
    assert 0 < st["device_ms"] <= st["mean_ms"] * st["completed"]


def _same_grid_models(k):
    """k problems of one grid and geometry with models of their own."""
    base = synth.small_case(n=(22, 20, 16), pml=6, nt=70, seed=60, shot_idx=[(11, 10, 2)])
    out = []
    for q in range(k):
        vp, vs, rho = synth.gardner(synth.layered_vp(base.nx, base.ny, base.nz, 61 + q, n_layers=3, vmin=2000,
                                                     vmax=3000))
        out.append(dataclasses.replace(base, vp=vp, vs=vs, rho=rho, seed=61 + q))
    return out


def test_pooled_contexts_give_the_results_of_new_ones():
    """Requests of one shape with different models run on pooled contexts
    (only the model and geometry are uploaded again): each result equals
    that of a new context of its own, the 16-bit-store requests included,
    and the server counts the reuse."""
    models = _same_grid_models(4)
    plan = [(m, k, p) for m in models for k, p in ((jv.JOB_RTM, jv.JV_FP32), (jv.JOB_FORWARD, jv.JV_FP32),
                                                   (jv.JOB_RTM, jv.JV_FP16))]
    want = [_alone(m, k, precision=p) for m, k, p in plan]
    with jv.Server(slots=2, budget=1 << 30) as srv:
        subs = [srv.submit_survey(k, m, precision=p) for m, k, p in plan]
        for rid, _ in subs:
            assert srv.wait(rid, timeout=180.0) == jv.JV_OK
        st = srv.stats()
    for (m, k, _), (_, got), w in zip(plan, subs, want):
        _check_same(k, got, w)
    # three shapes (RTM FP32, forward, RTM FP16), at most two contexts of each
    assert st["reused"] >= len(plan) - 6 and st["pooled"] <= 6


def test_idle_contexts_give_way_to_other_shapes():
    """A budget that holds one context at a time: alternating shapes must
    release the idle pooled context of the other shape before creating
    their own, and every result is still that of a context of its own."""
    a = _cases()[0]
    b = _cases()[2]
    fa = jv.footprint(a.nx, a.ny, a.nz, a.pml, a.nt, a.rec_width, jv.JOB_RTM, n_recv=len(a.recvs))
    fb = jv.footprint(b.nx, b.ny, b.nz, b.pml, b.nt, b.rec_width, jv.JOB_RTM, n_recv=len(b.recvs))
    want = {id(a): _alone(a, jv.JOB_RTM), id(b): _alone(b, jv.JOB_RTM)}
    with jv.Server(slots=2, budget=max(fa, fb) + min(fa, fb) // 2) as srv:
        for s in (a, b, a, b, a):
            rid, got = srv.submit_survey(jv.JOB_RTM, s)
            assert srv.wait(rid, timeout=180.0) == jv.JV_OK
            _check_same(jv.JOB_RTM, got, want[id(s)])
            st = srv.stats()
            assert st["pooled"] == 1 and st["bytes_in_use"] <= st["budget"]


@pytest.mark.parametrize("precision", [jv.JV_FP16, jv.JV_BF16])
def test_request_boundary_store_precision(precision):
    """A request's own boundary-store precision reaches its context: a
    16-bit-store request next to an FP32 one gives the images of a context
    with that store, and they differ from the FP32 store's (the replayed rim
    is rounded), within the 16-bit store's image error."""
    cases = _cases()
    w16 = _alone(cases[0], jv.JOB_RTM, precision=precision)
    w32 = _alone(cases[0], jv.JOB_RTM)
    with jv.Server(slots=2, budget=1 << 30) as srv:
        a = srv.submit_survey(jv.JOB_RTM, cases[0], precision=precision)
        b = srv.submit_survey(jv.JOB_RTM, cases[0])
        for rid, _ in (a, b):
            assert srv.wait(rid, timeout=180.0) == jv.JV_OK
    _check_same(jv.JOB_RTM, a[1], w16)
    _check_same(jv.JOB_RTM, b[1], w32)
    assert any(not np.array_equal(a[1][q], b[1][q]) for q in range(5))
    assert max(rel_l2(a[1][q], b[1][q]) for q in range(5)) <= 1e-3


def test_concurrent_grids_of_different_stage_sizes():
    """Requests whose full-gridext stress kernel needs different shared
    memory (other x widths and absorbing widths) running side by side."""
    cases = [synth.small_case(n=(22, 20, 16), pml=6, nt=60, seed=41),
             synth.small_case(n=(60, 14, 12), pml=8, nt=60, seed=42),
             synth.small_case(n=(96, 10, 10), pml=10, nt=60, seed=43)]
    plan = [(c, k) for c in cases for k in (jv.JOB_FORWARD, jv.JOB_RTM)] * 2
    want = {(id(c), k): _alone(c, k) for c, k in plan[:6]}
    with jv.Server(slots=6, budget=1 << 32) as srv:
        subs = [srv.submit_survey(k, c) for c, k in plan]
        for rid, _ in subs:
            assert srv.wait(rid, timeout=180.0) == jv.JV_OK
    for (c, k), (_, got) in zip(plan, subs):
        _check_same(k, got, want[(id(c), k)])


def test_budget_holds_while_requests_run():
    s = _cases()[0]
    one = jv.footprint(s.nx, s.ny, s.nz, s.pml, s.nt, s.rec_width, jv.JOB_RTM, n_recv=len(s.recvs))
    with jv.Server(slots=4, budget=one + one // 2) as srv:  # room for one request at a time
        subs = [srv.submit_survey(jv.JOB_RTM, s) for _ in range(4)]
        t0 = time.time()
        while srv.stats()["completed"] < 4 and time.time() - t0 < 180.0:
            st = srv.stats()
            assert st["bytes_in_use"] <= st["budget"]
            assert st["running"] <= 1
            time.sleep(0.002)
        for rid, _ in subs:
            assert srv.wait(rid, timeout=60.0) == jv.JV_OK
    want = _alone(s, jv.JOB_RTM)
    for _, got in subs:
        _check_same(jv.JOB_RTM, got, want)


def test_footprint_covers_what_a_context_allocates():
    for s in _cases():
        with jv.Context.from_survey(s) as ctx:
            obs = ctx.forward(0)
            ctx.rtm_shot(0, obs)
            held = ctx.info().device_bytes
        est = jv.footprint(s.nx, s.ny, s.nz, s.pml, s.nt, s.rec_width, jv.JOB_RTM, n_recv=len(s.recvs))
        assert held <= est <= 1.3 * held + (4 << 20), (s.name, held, est)


def test_cancel_and_timeout():
    big = synth.small_case(n=(48, 44, 40), pml=8, nt=1500, seed=14)
    small = _cases()[0]
    with jv.Server(slots=1, budget=1 << 31) as srv:
        first, _ = srv.submit_survey(jv.JOB_RTM, big)
        second, _ = srv.submit_survey(jv.JOB_FORWARD, small)
        with pytest.raises(jv.JvError) as e:  # a bounded wait on an unfinished request
            srv.wait(first, timeout=0.0)
        assert e.value.code == jv.JV_ETIMEOUT
        srv.cancel(second)
        assert srv.poll(second) == (jv.JOB_CANCELLED, jv.JV_ECANCELED)
        with pytest.raises(jv.JvError) as e:  # a running request cannot be cancelled
            while srv.poll(first)[0] == jv.JOB_QUEUED:
                time.sleep(0.001)
            srv.cancel(first)
        assert e.value.code == jv.JV_ESTATE
        assert srv.wait(first, timeout=180.0) == jv.JV_OK
        st = srv.stats()
        assert st["cancelled"] == 1 and st["completed"] == 1
