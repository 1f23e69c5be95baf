"""Receiver FK true-amplitude / deghost spreading (Receiver::spread_sdomain,
and spread_kdomain) on the GPU through the C ABI against the CPU
restatements: receivers off the grid nodes, obliquity and deghost on and off,
both sides, the low-cut ramp, even and odd FFT lengths, a line (ny = 1) and a
grid, the k-domain ghost threshold with and without its scaling.  FP32
cuFFT / cuBLAS against float64 sums: 1e-5 (rel. L2)."""
import numpy as np
import pytest

from konglong_b200.propagator import fk_spread
from oracle import fk_oracle as F
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

CASES = [
    # nx, ny, nt, ntfft, trueamp, deghost, side, flcut, flpass, kdomain, fmax
    (24, 20, 100, 160, 1, 0, -1, 0.0, 0.0, False, 0.0),
    (24, 20, 100, 160, 1, 1, -1, 3.0, 8.0, False, 0.0),
    (24, 20, 100, 165, 0, 1, 1, 0.0, 5.0, False, 0.0),
    (40, 1, 120, 180, 1, 1, -1, 2.0, 6.0, False, 0.0),
    (24, 20, 100, 160, 1, 1, -1, 3.0, 8.0, True, 10.0),   # threshold scaled (k z at fmax < pi / 2)
    (24, 20, 100, 165, 0, 1, 1, 0.0, 5.0, True, 40.0),
    (40, 1, 120, 180, 1, 0, -1, 0.0, 0.0, True, 40.0),
]


@pytest.mark.parametrize("case", CASES)
def test_fk_spread_matches_restatement(case):
    nx, ny, nt, ntfft, trueamp, deghost, side, flcut, flpass, kdomain, fmax = case
    rng = np.random.default_rng(nx + ny + ntfft)
    nr = 30
    xy = np.stack([rng.uniform(0, nx - 1, nr), rng.uniform(0, ny - 1, nr) if ny > 1 else np.zeros(nr)], 1)
    t = np.arange(nt) * 0.004
    f0 = rng.uniform(8, 25, nr)
    traces = (np.sin(2 * np.pi * f0[:, None] * t[None, :]) * np.exp(-((t[None, :] - 0.15) / 0.05) ** 2)
              ).astype(np.float32)
    kw = dict(vsurf=1500.0, z=15.0, trueamp=trueamp, deghost=deghost, side=side, flcut=flcut, flpass=flpass)
    if kdomain:
        got = fk_spread(nx, ny, nt, ntfft, 0.004, 10.0, 10.0, xy, traces, kdomain=True, fmax=fmax, **kw)
        xy_m = xy.astype(np.float32) * np.float32(10.0)
        want = F.fk_deghost_kdomain(nx, ny, nt, ntfft, 0.004, 10.0, 10.0, xy_m, traces, fmax=fmax, **kw)
    else:
        got = fk_spread(nx, ny, nt, ntfft, 0.004, 10.0, 10.0, xy, traces, **kw)
        want = F.fk_deghost(nx, ny, nt, ntfft, 0.004, 10.0, 10.0, xy, traces, **kw)
    assert np.abs(want).max() > 0
    assert rel_l2(got, want) < 1e-5


@pytest.mark.parametrize("kdomain", [False, True])
def test_fk_spread_edges(kdomain):
    """No receivers gives a zero grid; receivers on the last grid node and at
    the origin are accepted and match the restatement."""
    nx, ny, nt, ntfft = 20, 12, 64, 96
    z = fk_spread(nx, ny, nt, ntfft, 0.004, 10.0, 10.0, np.zeros((0, 2), np.float32), np.zeros((0, nt), np.float32),
                  1500.0, 10.0, kdomain=kdomain)
    assert z.shape == (ny, nx, nt) and not np.any(z)
    xy = np.array([[nx - 1, ny - 1], [0.0, 0.0], [7.25, 3.5]], np.float32)
    t = np.arange(nt) * 0.004
    traces = np.stack([np.sin(2 * np.pi * f * t) * np.exp(-((t - 0.1) / 0.03) ** 2) for f in (12, 18, 25)]
                      ).astype(np.float32)
    kw = dict(vsurf=1500.0, z=10.0, trueamp=1, deghost=1, side=-1)
    got = fk_spread(nx, ny, nt, ntfft, 0.004, 10.0, 10.0, xy, traces, kdomain=kdomain, fmax=40.0, **kw)
    if kdomain:
        want = F.fk_deghost_kdomain(nx, ny, nt, ntfft, 0.004, 10.0, 10.0, xy * np.float32(10.0), traces, fmax=40.0,
                                    **kw)
    else:
        want = F.fk_deghost(nx, ny, nt, ntfft, 0.004, 10.0, 10.0, xy, traces, **kw)
    assert np.abs(want).max() > 0
    assert rel_l2(got, want) < 1e-5
