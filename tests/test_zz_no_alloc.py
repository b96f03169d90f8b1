"""jv_forward_noalloc: forward modelling that allocates no device memory.

It exists for callers that cannot call cudaMalloc when they model a shot
(a memory pool that already owns the free device memory, or a path where an
allocation could block), so it takes every input and output as device
memory and carves its working memory out of a fixed array compiled into
libjv.  This file is collected last so that a run stopping at the first
failure has already run every other test.

Checked here, through the C ABI: two calls in a row give the traces of the
allocating context path (jv_create + jv_forward) within the trace tolerance
of the parity tests (2e-5 relative L2), the second call leaves the device's
free memory unchanged, the same holds on a caller's non-blocking stream, and
a problem too large for the array is refused.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import pkg, rel_l2

jv = pkg()
pytestmark = pytest.mark.gpu


def _run(s, out, nkept, stream=None):
    import torch

    L = jv.lib()
    dev = out.device
    vp = torch.from_numpy(np.ascontiguousarray(s.vp)).to(dev)
    vs = torch.from_numpy(np.ascontiguousarray(s.vs)).to(dev)
    rho = torch.from_numpy(np.ascontiguousarray(s.rho)).to(dev)
    g = jv.Grid(s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz)
    src = np.ascontiguousarray(s.shots[0], dtype=np.float32)
    rec = np.ascontiguousarray(s.recvs, dtype=np.float32)
    fp = C.POINTER(C.c_float)
    torch.cuda.synchronize()
    rc = L.jv_forward_noalloc(C.byref(g), C.c_void_p(vp.data_ptr()), C.c_void_p(vs.data_ptr()),
                              C.c_void_p(rho.data_ptr()), s.dt, s.fm, s.nt, src.ctypes.data_as(fp), rec.shape[0],
                              rec.ctypes.data_as(fp), C.c_void_p(out[0].data_ptr()), C.c_void_p(out[1].data_ptr()),
                              C.c_void_p(out[2].data_ptr()), C.byref(nkept), stream)
    torch.cuda.synchronize()
    return rc


def test_noalloc_matches_context_path_on_two_calls(synth):
    import torch

    s = synth.small_case(n=(40, 36, 30), pml=8, nt=200, seed=31, nrec=60)
    with jv.Context.from_survey(s) as ctx:
        ref = ctx.forward(0)
    out = torch.empty((3, s.recvs.shape[0], s.nt), dtype=torch.float32, device="cuda:0")
    nkept = C.c_int(-1)
    for call in range(2):
        out.fill_(float("nan"))  # stale results of the first call must not pass the second
        free0 = torch.cuda.mem_get_info(0)[0]
        rc = _run(s, out, nkept)
        free1 = torch.cuda.mem_get_info(0)[0]
        assert rc == jv.JV_OK, jv.lib().jv_last_error()
        assert nkept.value == ref[0].shape[0]
        if call == 1:
            assert free1 == free0, (free0, free1)
        got = out[:, :nkept.value].cpu().numpy()
        for a, b in zip(got, ref):
            assert np.all(np.isfinite(a))
            assert rel_l2(a, b) <= 2e-5, (call, rel_l2(a, b))


def test_noalloc_on_a_non_blocking_stream(synth):
    """The copies, clears and kernels all go on the caller's stream: on a
    non-blocking stream (no implicit ordering with the legacy stream) the
    traces still match the context path, on two calls in a row."""
    import torch

    s = synth.small_case(n=(36, 32, 28), pml=8, nt=160, seed=33, nrec=40)
    with jv.Context.from_survey(s) as ctx:
        ref = ctx.forward(0)
    out = torch.empty((3, s.recvs.shape[0], s.nt), dtype=torch.float32, device="cuda:0")
    nkept = C.c_int(-1)
    st = torch.cuda.Stream(device=0)
    for call in range(2):
        out.fill_(float("nan"))
        rc = _run(s, out, nkept, stream=C.c_void_p(st.cuda_stream))
        assert rc == jv.JV_OK, jv.lib().jv_last_error()
        got = out[:, :nkept.value].cpu().numpy()
        for a, b in zip(got, ref):
            assert np.all(np.isfinite(a))
            assert rel_l2(a, b) <= 2e-5, (call, rel_l2(a, b))


def test_noalloc_refuses_problems_larger_than_its_array(synth):
    import torch

    s = synth.small_case(n=(90, 90, 90), pml=10, nt=4, seed=32, nrec=4)
    out = torch.empty((3, 4, 4), dtype=torch.float32, device="cuda:0")
    nkept = C.c_int(-1)
    rc = _run(s, out, nkept)
    assert rc == jv.JV_EINVAL
    assert b"MiB" in jv.lib().jv_last_error()
