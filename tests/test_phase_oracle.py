"""The phase-correction oracle (PhaseCorrection, bgprtm/PhaseCorrection.cpp)
on the CPU against closed-form answers: a dispersion-free table returns its
band-limited input, a tone through the dispersion table drifts in phase by
(t - t0) dsp(w) per sample (sin and acos forms), resampling and output time
shifts move a periodic signal as the phase formulas say, the constant phase
rotation and the w_pow factor act per bin, and the routing of applyForward /
applyBackward refuses what the reference asserts against; plus the C ABI's
argument checks, which return before any device work."""
import ctypes as C
import math

import numpy as np
import pytest

from konglong_b200 import _lib
from konglong_b200.propagator import PhaseArgs, pad_fft_length
from oracle import phase_oracle as P


def _periodic(n, bins, rng, sine=False):
    t = np.arange(n)
    x = np.zeros(n)
    for k in bins:
        a, ph = rng.standard_normal(), rng.uniform(0, 2 * np.pi)
        x += a * (np.sin if sine else np.cos)(2 * np.pi * k * t / n + ph)
    return x


def test_dispersion_free_table_returns_the_band_limited_input():
    rng = np.random.default_rng(1)
    nt, ntfft, dt = 300, 480, 0.004
    x = rng.standard_normal((4, nt))
    x -= np.outer((x * (-1.0) ** np.arange(nt)).sum(1) / nt, (-1.0) ** np.arange(nt))  # no Nyquist part
    p = P.Plan(nt, dt, 0.0, 0.0, 1.0 / (2 * dt), P.BWD, ntfft=ntfft)  # fmax = Nyquist: every bin in the band
    assert p.nw1 == p.nw
    np.testing.assert_allclose(P.apply_backward(p, x), x, atol=2e-5 * np.abs(x).max())


@pytest.mark.parametrize("ratio", [0.0, 1.0, 0.5])
def test_tone_drifts_by_the_dispersion_phase(ratio):
    n, dt, Dt, k0 = 256, 0.002, 0.002, 23
    x = np.cos(2 * np.pi * k0 * np.arange(n) / n)[None, :]
    p = P.Plan(n, dt, Dt, 0.01, 120.0, P.BWD, ntfft=n, tdsp_acos_ratio=ratio)  # w Dt <= 1.51 in the band
    w = k0 * 2 * math.pi / (n * dt)
    xx = w * Dt
    dsp = (ratio * (math.acos(1 - 0.5 * xx * xx) - xx) + (1 - ratio) * (xx - 2 * math.sin(xx / 2))) * dt / Dt
    it = np.arange(n)
    it0 = 0.01 / dt
    want = np.cos(2 * np.pi * k0 * it / n - (it - it0) * dsp)
    assert abs(dsp) > 1e-3
    np.testing.assert_allclose(P.apply_backward(p, x)[0], want, atol=3e-4)


@pytest.mark.parametrize("dt_out", [0.002, 0.0013])
def test_resampling_evaluates_the_band_limited_trace_on_the_new_samples(dt_out):
    n, dt = 200, 0.004
    rng = np.random.default_rng(2)
    bins = [3, 11, 17]
    t = np.arange(n)
    amp, ph = rng.standard_normal(3), rng.uniform(0, 2 * np.pi, 3)
    f = lambda tt: sum(a * np.cos(2 * np.pi * k * tt / (n * dt) + q) for a, k, q in zip(amp, bins, ph))
    x = f(t * dt)[None, :]
    nt_out = int(n * dt / dt_out) - 1
    p = P.Plan(n, dt, 0.0, 0.0, 60.0, P.BWD, 0, 0, 1, nt_out, dt_out, ntfft=n)  # ExtractReceiverData:87's form
    np.testing.assert_allclose(P.apply_backward(p, x)[0], f(np.arange(nt_out) * dt_out), atol=2e-4 * np.abs(x).max())


def test_output_start_time_shifts_the_trace():
    n, dt = 240, 0.004
    x = _periodic(n, [5, 9, 30], np.random.default_rng(3), sine=True)
    shift = 3.5 * dt
    p = P.Plan(n, dt, 0.0, 0.0, 100.0, P.BWD, 0, 0, 1, n, dt, shift, ntfft=n)  # dt_out == dt: the integer-shift form
    # a periodic band-limited trace delayed by the shift, evaluated through its spectrum
    X = np.fft.rfft(x)
    k = np.arange(X.size)
    want = np.fft.irfft(X * np.exp(-2j * np.pi * k * shift / (n * dt)), n)
    np.testing.assert_allclose(P.apply_backward(p, x[None, :])[0], want, atol=2e-4 * np.abs(x).max())


def test_phase_rotation_and_w_pow_act_per_bin():
    n, dt, k0 = 128, 0.004, 9
    th = 2 * np.pi * k0 * np.arange(n) / n
    x = np.cos(th)[None, :]
    rot = P.Plan(n, dt, 0.0, 0.0, 1.0 / (2 * dt), P.BWD, 0.0, 90.0, do_tdsp=0, ntfft=n)
    np.testing.assert_allclose(P.apply_backward(rot, x)[0], -np.sin(th), atol=1e-6)
    flip = P.Plan(n, dt, 0.0, 0.0, 1.0 / (2 * dt), P.BWD, 0.0, 180.0, do_tdsp=0, ntfft=n)
    np.testing.assert_allclose(P.apply_backward(flip, x)[0], -x[0], atol=1e-6)
    der = P.Plan(n, dt, 0.0, 0.0, 1.0 / (2 * dt), P.BWD, 1.0, 0.0, do_tdsp=0, ntfft=n)
    w = k0 * 2 * np.pi / (n * dt)
    np.testing.assert_allclose(P.apply_backward(der, x)[0], w * x[0], rtol=0, atol=1e-5 * w)


def test_forward_dispersion_free_table_doubles_the_band():
    """dft_fft's table carries the factor 2 of the one-sided inverse sum; with
    the unnormalised full inverse transform (the inferred libfftv
    convention) a dispersion-free forward correction doubles the trace."""
    n, dt = 160, 0.004
    x = _periodic(n, [4, 13, 40], np.random.default_rng(4))[None, :]
    p = P.Plan(n, dt, 0.0, 0.0, 1.0 / (2 * dt), P.FWD, ntfft=n)
    np.testing.assert_allclose(P.apply_forward(p, x), 2 * x, atol=1e-4 * np.abs(x).max())


def test_routing_refusals_and_the_no_op():
    x = np.zeros((1, 50))
    with pytest.raises(ValueError):
        P.apply_forward(P.Plan(50, 0.004, 0.004, 0.0, 60.0, P.BWD, ntfft=80), x)
    with pytest.raises(ValueError):  # dft_fft cannot resample
        P.apply_backward(P.Plan(50, 0.004, 0.0, 0.0, 60.0, P.BWD, 0, 0, 1, 40, 0.005, ntfft=80,
                                tdsp_correction=1, transform=2), x)
    p = P.Plan(50, 0.004, 0.004, 0.0, 60.0, P.BWD, do_tdsp=0, ntfft=80)
    y = np.random.default_rng(5).standard_normal((2, 50))
    assert p.identity and np.array_equal(P.apply_backward(p, y), y)


def test_pad_fft_length():
    assert pad_fft_length(450) == 450 and pad_fft_length(451) == 480 and pad_fft_length(1) == 2
    assert pad_fft_length(1023) == 1024 and pad_fft_length(2 * 11 * 13) == 288


def test_capi_refusals_return_before_device_work():
    L = _lib.lib()
    good = dict(nt=50, dt=0.004, Dt=0.004, t0=0.0, fmax=60.0, direction=2, w_pow=0.0, phase_deg=0.0, do_tdsp=1,
                nt_out=-1, dt_out=-1.0, t0_out=0.0, ntfft=80, tdsp_correction=2, skip_tdsp_correction=0,
                tdsp_acos_ratio=0.0, skip_jacobian=0, transform=0)
    tr = np.zeros(50, np.float32)
    out = np.zeros(200, np.float32)
    cases = [(dict(ntfft=49), 2), (dict(ntfft=81), 2), (dict(dt=0.0), 2), (dict(direction=3), 2),
             (dict(transform=3), 2), (dict(Dt=-1.0), 2), (dict(fmax=-1.0), 2),
             (dict(), 1),                                               # applyForward needs FWD
             (dict(direction=1, nt_out=40, dt_out=0.005), 1),           # forward cannot resample
             (dict(nt_out=40, dt_out=0.005, tdsp_correction=1, transform=2), 2),  # dft_fft cannot resample
             (dict(do_tdsp=0, nt_out=40, dt_out=0.005), 2),             # the no-op cannot resample
             (dict(do_tdsp=0, phase_deg=10.0, nt_out=120, dt_out=0.001), 2),  # plain fft_dft: ntfft < nt_out
             (dict(), 0)]
    for b, apply in cases:
        a = PhaseArgs(**{**good, **b})
        assert L.rtm_phase_correct(C.byref(a), apply, 1, tr, out, 1.0) == -1, (b, apply)
    assert L.rtm_phase_correct(None, 2, 1, tr, out, 1.0) == -1
    a = PhaseArgs(**good)
    assert L.rtm_phase_correct(C.byref(a), 2, -1, tr, out, 1.0) == -1
