"""The FK true-amplitude / deghost spreading restatement on known answers
(CPU): one column, zero-mean trace, obliquity only -> the trace times
sqrt(ntfft) (the reference's scalar times an unnormalised round trip); a
cosine at a bin frequency through deghost -> the sine of the same frequency
times sqrt(ntfft) side / (2 sin(k z)); evanescent wavenumbers removed."""
import numpy as np

from oracle import fk_oracle as F


def test_vertical_obliquity_is_identity_up_to_the_scaling():
    nt = ntfft = 96
    tr = np.random.default_rng(1).standard_normal(nt)
    tr -= tr.mean()
    out = F.fk_deghost(1, 1, nt, ntfft, 0.004, 10.0, 10.0, [(0.0, 0.0)], [tr], 1500.0, 10.0, 1, 0)
    np.testing.assert_allclose(out[0, 0], np.sqrt(ntfft) * tr.astype(np.float32), rtol=0, atol=1e-5)


def test_deghost_known_answer():
    nt = ntfft = 128
    dt, v, z, m = 0.004, 1500.0, 12.0, 9
    t = np.arange(nt)
    tr = np.cos(2 * np.pi * m * t / ntfft)
    for side in (-1, 1):
        out = F.fk_deghost(1, 1, nt, ntfft, dt, 10.0, 10.0, [(0.0, 0.0)], [tr], v, z, 1, 1, side=side)
        k = 2 * np.pi * m / (dt * ntfft * v)
        want = -np.sqrt(ntfft) * side / (2 * np.sin(k * z)) * np.sin(2 * np.pi * m * t / ntfft)
        np.testing.assert_allclose(out[0, 0], want, rtol=0, atol=1e-4 * np.abs(want).max())


def test_evanescent_wavenumbers_are_removed():
    """A lateral wavelength shorter than the frequency allows (kx > w / v)
    is cut entirely; a long one passes."""
    nx, nt = 32, 64
    dx, dt, v = 10.0, 0.004, 1500.0
    t = np.arange(nt)
    w = np.cos(2 * np.pi * 4 * t / nt)           # 15.6 Hz -> k = 0.065 / m
    for kx_idx, passes in ((8, False), (1, True)):  # kx = 0.157 / m and 0.0196 / m
        lat = np.cos(2 * np.pi * kx_idx * np.arange(nx) / nx)
        xy = [(float(i), 0.0) for i in range(nx)]
        traces = [lat[i] * w for i in range(nx)]
        out = F.fk_deghost(nx, 1, nt, nt, dt, dx, 10.0, xy, traces, v, 0.0, 1, 0, khpass=0.49, khcut=0.5,
                           nlimit=1)
        energy = np.abs(out[0, 4:-4]).max()
        assert (energy > 1e-2) == passes, (kx_idx, energy)


def test_kdomain_equals_sdomain_on_grid_node_receivers():
    """With one receiver on every grid node, delta spread kernels and k tapers
    that pass every propagating wavenumber, the two forms filter the same
    grid data: spread_kdomain's phase-shift sums are then the DFT of
    spread_sdomain's grid."""
    nx, ny, nt, ntfft = 16, 12, 64, 96
    rng = np.random.default_rng(0)
    xy = [(float(i), float(j)) for j in range(ny) for i in range(nx)]
    t = np.arange(nt) * 0.004
    tr = np.array([np.sin(2 * np.pi * 15 * t) * np.exp(-((t - 0.1) / 0.03) ** 2) * rng.uniform(0.5, 1) for _ in xy],
                  np.float32)
    for trueamp, deghost in ((1, 0), (0, 1), (1, 1)):
        s = F.fk_deghost(nx, ny, nt, ntfft, 0.004, 10.0, 10.0, xy, tr, 1500.0, 10.0, trueamp, deghost, nlimit=1)
        k = F.fk_deghost_kdomain(nx, ny, nt, ntfft, 0.004, 10.0, 10.0, [(x * 10.0, y * 10.0) for x, y in xy], tr,
                                 1500.0, 10.0, trueamp, deghost, khpass=0.45, khcut=0.5, fmax=1000.0)
        assert np.abs(s - k).max() <= 1e-6 * np.abs(s).max()
