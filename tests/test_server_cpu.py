"""The request server without a GPU: footprint estimates (the admission
unit), argument checks, and the budget refusal, all decided on the host
before any request reaches a device."""
import numpy as np
import pytest

from conftest import pkg

jv = pkg()


def test_footprint_grows_with_the_problem():
    f = jv.footprint
    assert f(40, 40, 40, 10, 500, kind=jv.JOB_FORWARD) < f(60, 40, 40, 10, 500, kind=jv.JOB_FORWARD)
    assert f(40, 40, 40, 10, 500, kind=jv.JOB_FORWARD) < f(40, 40, 40, 10, 500, kind=jv.JOB_RTM)
    assert f(40, 40, 40, 10, 500, rec_width=1) < f(40, 40, 40, 10, 500, rec_width=4)
    assert f(40, 40, 40, 10, 500) < f(40, 40, 40, 10, 1000)          # the boundary store grows with nt
    assert f(40, 40, 40, 10, 500, n_recv=100) - f(40, 40, 40, 10, 500) == 3 * 100 * 500 * 4
    # cfg2 RTM: two 13-field wavefields of 240^3 cells plus a 6.7 GB boundary store
    b = f(200, 200, 200, 20, 2000)
    assert 8e9 < b < 11e9
    with pytest.raises(jv.JvError):
        f(4, 40, 40, 10, 500)


def test_server_refuses_request_beyond_budget(synth):
    s = synth.small_case(n=(24, 20, 18), pml=6, nt=100, seed=3)
    with jv.Server(slots=2, budget=1 << 20) as srv:  # 1 MiB: nothing fits
        with pytest.raises(jv.JvError) as e:
            srv.submit(jv.JOB_RTM, s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.vp, s.vs, s.rho, s.dt, s.fm, s.nt,
                       s.shots[0], s.recvs)
        assert e.value.code == jv.JV_ENOMEM and "budget" in str(e.value)
        st = srv.stats()
        assert st["submitted"] == 0 and st["budget"] == 1 << 20


def test_server_argument_checks():
    with pytest.raises(jv.JvError):
        jv.Server(slots=0, budget=1 << 30)
    with jv.Server(slots=1, budget=1 << 30) as srv:
        a = np.ones(10 * 10 * 10, np.float32)
        with pytest.raises(jv.JvError):  # grid below 8 cells
            srv.submit(jv.JOB_FORWARD, 4, 10, 10, 4, 1.0, 1.0, 1.0, a, a, a, 1e-3, 10.0, 10, (1, 1, 1),
                       np.zeros((1, 3), np.float32))
        with pytest.raises(jv.JvError):  # unknown kind
            srv.submit(7, 10, 10, 10, 4, 1.0, 1.0, 1.0, a, a, a, 1e-3, 10.0, 10, (1, 1, 1),
                       np.zeros((1, 3), np.float32))
        with pytest.raises(jv.JvError):
            srv.poll(12345)


def test_sixteen_bit_store_admitted_where_fp32_is_not(synth):
    """The server admits a request by its footprint with the boundary store
    it asks for: a budget one byte short of the FP32 request's footprint
    refuses it, and admits the same request with a 16-bit store."""
    s = synth.small_case(n=(24, 20, 18), pml=6, nt=2000, seed=3)
    args = (jv.JOB_RTM, s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.vp, s.vs, s.rho, s.dt, s.fm, s.nt, s.shots[0],
            s.recvs)
    need = jv.footprint(s.nx, s.ny, s.nz, s.pml, s.nt, kind=jv.JOB_RTM, n_recv=s.recvs.shape[0])
    with jv.Server(slots=1, budget=need - 1) as srv:
        with pytest.raises(jv.JvError) as e:
            srv.submit(*args)
        assert e.value.code == jv.JV_ENOMEM
        with pytest.raises(jv.JvError):  # not a jv_precision
            srv.submit(*args, precision=7)
        rid = srv.submit(*args, precision=jv.JV_FP16)
        assert rid > 0 and srv.stats()["submitted"] == 1
        # admitted: a worker takes it at once (without a GPU it fails there)
        srv.wait(rid, timeout=120.0)
