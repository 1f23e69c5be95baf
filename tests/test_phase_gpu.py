"""Phase correction on the GPU (rtm_phase_correct: PhaseCorrection,
bgprtm/PhaseCorrection.cpp) against the float64 restatement on the same
seeded traces, every route the reference's call sites and global parameters
reach: the source wavelet's forward correction (Source.cpp:150-151: dft_fft
with the table, sin Jacobian, dispersion), the receivers' backward
correction (ExtractReceiverData.cpp:369-373: fft_dft with the table), the
resample-and-shift form without dispersion (:87-90) and with it plus a
scaler (:101-105), the integer-shift form (dt_out == dt), acos / mixed
dispersion forms, the tdsp_correction 1 routes, the plain-transform routes
(no table) with w_pow and a phase rotation, and the no-op.  Sizes: one trace,
ragged counts around the 64-trace tiles, odd nt and nt_out.  Tolerance: the
table and the products are FP32 on both sides of the reference's own sums
(thousands of terms); measured worst relative L2 1.2e-6, held to 5e-6."""
import numpy as np
import pytest

from konglong_b200.propagator import PhaseCorrection
from oracle import phase_oracle as P
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _ricker_traces(ntr, nt, dt, seed, fpeak=25.0):
    rng = np.random.default_rng(seed)
    t = np.arange(nt) * dt
    out = np.zeros((ntr, nt), np.float32)
    for r in range(ntr):
        t0 = rng.uniform(0.1, 0.8) * nt * dt
        a = (np.pi * fpeak * (t - t0)) ** 2
        out[r] = (rng.uniform(0.5, 2.0) * (1 - 2 * a) * np.exp(-a)).astype(np.float32)
    out += (0.01 * rng.standard_normal(out.shape)).astype(np.float32)
    return out


def _check(kw, apply, ntr, nt, dt, seed, scaler=1.0):
    kw = dict(kw)
    ntfft = kw.pop("ntfft", None)
    pc = PhaseCorrection(nt, dt, *kw.pop("pos"), ntfft=ntfft, **kw)
    x = _ricker_traces(ntr, nt, dt, seed)
    pos = [pc.args.dt, pc.args.Dt, pc.args.t0, pc.args.fmax, pc.args.direction, pc.args.w_pow, pc.args.phase_deg,
           pc.args.do_tdsp, pc.args.nt_out, pc.args.dt_out, pc.args.t0_out]
    p = P.Plan(nt, *pos, ntfft=pc.args.ntfft, tdsp_correction=pc.args.tdsp_correction,
               skip_tdsp_correction=pc.args.skip_tdsp_correction, tdsp_acos_ratio=pc.args.tdsp_acos_ratio,
               skip_jacobian=bool(pc.args.skip_jacobian), transform=pc.args.transform)
    if apply == 1:
        got, want = pc.applyForward(x, ntr), P.apply_forward(p, x)
    else:
        got, want = pc.applyBackward(x, ntr, scaler), P.apply_backward(p, x, scaler, pc.args.nt_out)
    assert got.shape == want.shape and np.isfinite(got).all()
    assert np.abs(want).max() > 0
    return got, want


FWD, BWD = PhaseCorrection.FWD, PhaseCorrection.BWD
DT, DTP = 0.004, 0.001  # data sample interval, propagation dt
ROUTES = {
    "source_fwd": (dict(pos=(DTP, 0.05, 60.0, FWD)), 1),
    "source_fwd_wpow_phase": (dict(pos=(DTP, 0.05, 60.0, FWD, 1.0, 30.0)), 1),
    "source_fwd_no_jacobian": (dict(pos=(DTP, 0.0, 60.0, FWD), skip_jacobian=True), 1),
    "receiver_bwd": (dict(pos=(DTP, 0.0, 60.0, BWD)), 2),
    "receiver_bwd_acos": (dict(pos=(DTP, 0.0, 60.0, BWD), tdsp_acos_ratio=1.0), 2),
    "receiver_bwd_mixed": (dict(pos=(DTP, 0.02, 60.0, BWD), tdsp_acos_ratio=0.5), 2),
    "receiver_bwd_skip": (dict(pos=(DTP, 0.0, 60.0, BWD), skip_tdsp_correction=2), 2),
    "resample_no_dispersion": (dict(pos=(0.0, 0.0, 60.0, BWD, 0.0, 0.0, 1, 517, 0.0017)), 2),
    "resample_dispersion": (dict(pos=(DTP, 0.0, 60.0, BWD, 0.0, 0.0, 1, 301, 0.006, 0.01)), 2),
    "shift_same_dt": (dict(pos=(DTP, 0.0, 60.0, BWD, 0.0, 0.0, 1, 400, DT, 0.0138)), 2),
    "fwd_forced_fftdft_tdsp1": (dict(pos=(DTP, 0.02, 60.0, FWD), tdsp_correction=1, transform=1), 1),
    "bwd_forced_dftfft_tdsp1": (dict(pos=(DTP, 0.0, 60.0, BWD), tdsp_correction=1, transform=2), 2),
    "bwd_plain_wpow_phase": (dict(pos=(DTP, 0.0, 80.0, BWD, 2.0, -45.0, 0)), 2),
    "fwd_plain_phase": (dict(pos=(DTP, 0.0, 80.0, FWD, 0.0, 90.0, 0)), 1),
    "bwd_plain_resample": (dict(pos=(DTP, 0.0, 125.0, BWD, 0.5, 10.0, 0, 350, 0.004, 0.008)), 2),
}


@pytest.mark.parametrize("route", sorted(ROUTES))
@pytest.mark.parametrize("ntr,nt", [(1, 400), (67, 333), (130, 1001)])
def test_routes_match_the_oracle(route, ntr, nt):
    kw, apply = ROUTES[route]
    got, want = _check(kw, apply, ntr, nt, DT, seed=ntr + nt)
    assert rel_l2(got, want) < 5e-6, (route, rel_l2(got, want))


def test_scaler_on_the_first_nt_out_samples():
    kw = dict(pos=(DTP, 0.0, 60.0, BWD, 0.0, 0.0, 1, 301, 0.006))
    got, want = _check(kw, 2, 5, 500, DT, seed=7, scaler=1.0 / 12.5)
    assert rel_l2(got, want) < 5e-6
    unscaled, _ = _check(kw, 2, 5, 500, DT, seed=7)
    np.testing.assert_allclose(got, unscaled / 12.5, rtol=1e-6, atol=1e-7 * np.abs(unscaled).max())


def test_no_op_returns_the_input_bit_for_bit():
    pc = PhaseCorrection(300, DT, DTP, 0.0, 60.0, BWD, do_tdsp=0)
    x = _ricker_traces(4, 300, DT, 3)
    assert np.array_equal(pc.applyBackward(x, 4), x)
    fwd = PhaseCorrection(300, DT, DTP, 0.0, 60.0, FWD, do_tdsp=0)
    assert np.array_equal(fwd.applyForward(x, 4), x)


def test_large_batch_and_long_traces():
    """2000 traces of 3000 samples (the product kernel over many tiles) and a
    size-independent property: the traces go through independently, so the
    first trace matches its own one-trace call (the product sums are the
    same; the batched transform may take another algorithm)."""
    pc = PhaseCorrection(3000, DT, DTP, 0.0, 60.0, BWD)
    x = _ricker_traces(2000, 3000, DT, 11)
    got = pc.applyBackward(x, 2000)
    one = pc.applyBackward(x[:1], 1)
    assert rel_l2(got[:1], one) < 1e-6
    p = P.Plan(3000, DT, DTP, 0.0, 60.0, BWD, ntfft=pc.args.ntfft)
    idx = np.arange(0, 2000, 97)
    want = P.apply_backward(p, x[idx])
    assert rel_l2(got[idx], want) < 5e-6, rel_l2(got[idx], want)
