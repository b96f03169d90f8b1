"""Unit checks of the oracle's building blocks against the reference's
published constants and formulas."""
import math

import numpy as np


def test_diff_coeff_known_values(oracle):
    # staggered Taylor coefficients, jarvis_device_geometry_bones.hpp:29-49
    np.testing.assert_allclose(oracle.diff_coeff(4), [1.1962890625, -0.0797526041666667, 0.0095703125,
                                                      -0.000697544642857143], rtol=1e-12)
    np.testing.assert_allclose(oracle.diff_coeff(2), [1.125, -1.0 / 24.0], rtol=1e-12)
    np.testing.assert_allclose(oracle.diff_coeff(1), [1.0])
    for o in range(1, 5):
        c = oracle.diff_coeff(o)
        # consistency: sum (2r+1) c_r == 1 (first derivative exact on linears)
        assert abs(sum((2 * r + 1) * c[r] for r in range(o)) - 1.0) < 1e-12


def test_ntime_and_ricker(oracle):
    assert oracle.ntime(np.float32(0.3995), np.float32(1e-3)) == 400
    assert oracle.ntime(np.float32(0.16), np.float32(1e-4)) == 1600
    w = oracle.ricker(200, 25.0, 1e-3)
    n0 = int(math.floor(np.float32(1.3 / 25.0) / np.float32(1e-3) + 0.5))
    assert np.argmax(w) == n0
    assert abs(w[n0] - 1e4) < 1e-2
    t = (np.arange(200) - n0) * np.float32(1e-3)
    a = np.pi * 25.0 * t.astype(np.float32).astype(np.float64)
    np.testing.assert_allclose(w, (1e4 * (1 - 2 * a * a) * np.exp(-a * a)).astype(np.float32), rtol=0, atol=1e-3)


def test_gap_num(oracle):
    assert oracle.gap_num(-50.0, 75.0, 5.0) == 25
    assert oracle.gap_num(0.0, 0.0, 10.0) == 0
    assert oracle.gap_num(-80.0, 290.0, 10.0) == 37


def test_cpml_profile_sides(oracle):
    n, m, vp, d, fm = 60, 10, 3000.0, 10.0, 20.0
    dt = float(np.float32(1e-3))  # the reference's dt is a float
    N = m - 2
    # outer rim and interior: inactive (a=0, b=1)
    for c in (0, 1, n - 2, n - 1, m, n // 2, n - m - 1):
        act, ab = oracle.cpml_ab(c, n, m, vp, d, fm, dt)
        assert not act and ab[0] == 0.0 and ab[1] == 1.0
    # low side: s = m - c at integer nodes, m - c - 0.5 at half nodes
    act, ab = oracle.cpml_ab(2, n, m, vp, d, fm, dt)
    temp = 3.0 * 7.0 * vp / (2 * N * d)
    dd = temp * (N / N) ** 2
    b = math.exp(-(dd + math.pi * fm * 0.0) * dt)
    assert act and abs(ab[1] - b) < 1e-12 and abs(ab[0] - dd * (b - 1) / dd) < 1e-9
    # high side mirrors with integer/half swapped: integer at c=n-m is s=0.5
    act, ab = oracle.cpml_ab(n - m, n, m, vp, d, fm, dt)
    s = 0.5
    dd = temp * (s / N) ** 2
    al = math.pi * fm * (1 - s / N)
    assert act and abs(ab[1] - math.exp(-(dd + al) * dt)) < 1e-12
    # damping grows towards the outer edge on both sides
    lo = [oracle.cpml_ab(c, n, m, vp, d, fm, dt)[1][1] for c in range(2, m)]
    hi = [oracle.cpml_ab(c, n, m, vp, d, fm, dt)[1][1] for c in range(n - m, n - 2)]
    assert all(np.diff(lo) > 0) and all(np.diff(hi) < 0)


def test_forward_fp32_close_to_fp64(oracle, synth):
    s = synth.small_case(n=(16, 14, 12), pml=5, nt=80)
    p = oracle.Problem(s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.dt, s.fm, s.T, 1, s.shots, s.recvs, s.vp,
                       s.vs, s.rho)
    a = oracle.forward(p)
    b = oracle.forward(p, precision="f32")
    for x, y in zip(a, b):
        assert np.linalg.norm(x - y) / np.linalg.norm(x) < 1e-5


def test_rtm_reconstruction_w4_exact_order(oracle, synth):
    """rec_width 4 keeps the full 8th order at the rim: reconstruction is
    the exact time reverse up to rounding; rec_width 1 is approximate."""
    errs = {}
    for w in (1, 4):
        s = synth.small_case(n=(18, 16, 14), pml=6, nt=100, rec_width=w)
        p = oracle.Problem(s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.dt, s.fm, s.T, w, s.shots, s.recvs,
                           s.vp, s.vs, s.rho)
        tr = oracle.forward(p)
        _, errs[w] = oracle.rtm_shot(p, tr, want_recon=True)
    assert errs[4] < 1e-9, errs
    assert errs[1] < 0.2 and errs[1] > errs[4]


def test_store16_study_error(oracle, synth):
    """16-bit wavefield storage, emulated on the oracle (FP32 arithmetic,
    per-plane power-of-two scales), against plain FP32 storage: on a small
    RTM shot FP32 storage stays within 1e-4 of the FP64 oracle, while FP16
    and BF16 storage already exceed the 1e-3 image bound."""
    s = synth.small_case(n=(20, 18, 16), pml=6, nt=120, seed=3)
    p = oracle.Problem(s.nx, s.ny, s.nz, s.pml, s.dx, s.dy, s.dz, s.dt, s.fm, s.T, 1, s.shots, s.recvs, s.vp,
                       s.vs, s.rho)
    obs = oracle.forward(p)
    ref = oracle.rtm_shot(p, obs)

    def err(kind):
        with oracle.store16(kind):
            img = oracle.rtm_shot(p, obs, precision="f32")
        return max(float(np.linalg.norm(img[k] - ref[k]) / np.linalg.norm(ref[k])) for k in ref)

    e32, e16, eb16 = err("f32"), err("fp16"), err("bf16")
    assert e32 <= 1e-4, e32
    assert e16 > 1e-3, e16
    assert eb16 > e16, (eb16, e16)
    # the setting does not outlive the context
    img = oracle.rtm_shot(p, obs, precision="f32")
    assert max(float(np.linalg.norm(img[k] - ref[k]) / np.linalg.norm(ref[k])) for k in ref) <= 1e-4
