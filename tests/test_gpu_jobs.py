"""The job queue (jv_submit / jv_poll / jv_wait / jv_cancel) and the batch
call (jv_rtm_batch) on the GPU: the same traces and stacks as the direct
calls, queued jobs that can be cancelled, a bounded host wait that ends
with JV_ETIMEOUT, and JV_ESTATE for direct calls while jobs are pending.
Nothing here waits on the GPU without a limit: the only waits are host
waits with timeouts."""
import numpy as np
import pytest

from conftest import pkg, rel_l2

pytestmark = pytest.mark.gpu

jv = pkg()


def _case(synth, nt=60):
    return synth.small_case(n=(18, 16, 14), pml=5, nt=nt, seed=6, shot_idx=[(4, 5, 2), (12, 9, 3), (9, 9, 9)])


def test_jobs_match_direct_calls(synth):
    s = _case(synth)
    with jv.Context.from_survey(s) as ctx:
        obs = [ctx.forward(i) for i in range(3)]
        ctx.image_reset()
        for i in range(3):
            ctx.rtm_shot(i, obs[i])
        direct = ctx.images()

        ctx.image_reset()
        out = [np.zeros_like(obs[1][q]) for q in range(3)]
        ids = [ctx.submit(jv.JOB_RTM, 0, obs=obs[0]),
               ctx.submit(jv.JOB_FORWARD, 1, out=out),
               ctx.submit(jv.JOB_RTM, 1),            # models its own traces first
               ctx.submit(jv.JOB_RTM, 2, obs=obs[2])]
        for i in ids:
            assert ctx.wait(i, timeout=120.0) == jv.JV_OK
            assert ctx.poll(i) == (jv.JOB_DONE, jv.JV_OK)
        served = ctx.images()
    for q in range(3):
        assert np.array_equal(out[q], obs[1][q])
    for k in direct:
        assert rel_l2(served[k], direct[k]) <= 1e-12, k


def test_batch_matches_direct_calls(synth):
    s = _case(synth)
    with jv.Context.from_survey(s) as ctx:
        obs = [ctx.forward(i) for i in range(3)]
        ctx.image_reset()
        for i in (2, 0, 1):
            ctx.rtm_shot(i, obs[i])
        direct = ctx.images()
        ctx.image_reset()
        ctx.rtm_batch([2, 0, 1], [obs[2], obs[0], obs[1]])
        batched = ctx.images()
        assert ctx.last_ms() > 0
    for k in direct:
        assert rel_l2(batched[k], direct[k]) <= 1e-12, k


def test_cancel_timeout_and_busy(synth):
    s = _case(synth, nt=400)
    with jv.Context.from_survey(s) as ctx:
        ids = [ctx.submit(jv.JOB_RTM, i % 3) for i in range(6)]
        # the last one is still queued behind five migrations
        ctx.cancel(ids[-1])
        assert ctx.poll(ids[-1]) == (jv.JOB_CANCELLED, jv.JV_ECANCELED)
        states = [ctx.poll(i)[0] for i in ids[:-1]]
        if any(st in (jv.JOB_QUEUED, jv.JOB_RUNNING) for st in states):
            with pytest.raises(jv.JvError) as e:
                ctx.forward(0)
            assert e.value.code == jv.JV_ESTATE
        pending = [i for i in ids[:-1] if ctx.poll(i)[0] in (jv.JOB_QUEUED, jv.JOB_RUNNING)]
        if pending:
            with pytest.raises(jv.JvError) as e:
                ctx.wait(pending[-1], timeout=0.0)
            assert e.value.code == jv.JV_ETIMEOUT
        for i in ids[:-1]:
            assert ctx.wait(i, timeout=300.0) == jv.JV_OK
        with pytest.raises(jv.JvError) as e:
            ctx.cancel(ids[0])  # already done
        assert e.value.code == jv.JV_ESTATE
        ctx.forward(0)  # idle again


def test_failed_job_reports_its_error(synth):
    s = _case(synth)
    with jv.Context.from_survey(s) as ctx:
        with pytest.raises(jv.JvError):
            ctx.submit(jv.JOB_RTM, 7)  # no such shot: refused at submission
        ctx.set_geometry(np.array([[1e6, 0, 0]], np.float32), s.recvs)  # the shot now lies outside gridphy
        jid = ctx.submit(jv.JOB_FORWARD, 0, out=[None, None, None])
        assert ctx.wait(jid, timeout=60.0) == jv.JV_EINVAL
        st, res = ctx.poll(jid)
        assert st == jv.JOB_DONE and res == jv.JV_EINVAL
        assert "outside gridphy" in jv.lib().jv_last_error().decode()
