"""CPU restatement of the INVERSION imaging condition - test infrastructure (the
checker of the CUDA path, never the product).

ImagingCorrelator::inversion1 with derive / lapx / lapy / lapz
(bgprtm/ImagingCorrelator.cpp:195-278, 374-424) and the wavenumber convention of
assignW (:157-166): for volumes S, R of shape (ny, nx, nz) (z fastest)

    image += S R - dz(S) dz(R) - dx(S) dx(R) - dy(S) dy(R)    (dy only when ny > 1)

with d_a(f) = F^-1[ i (k_a / |k|) F[f] ], zero where |k| <= 1e-25, k[i] = -i dk for
i <= n/2 and (n - i) dk above, dk = 2 pi / (d n); F unnormalised forward, F^-1
normalised (the reference's 1/sqrt(N) on both sides).  Each derivative is taken
from the original spectrum (the reference overwrites the spectrum by the x
derivative when it has no y double grid; see the design notes).  Float64.
Parity: restated from the reference's sources, not run against them (the
correlator needs FFTW and the absent libCommon)."""
import numpy as np


def _k(n, d):
    dk = 2.0 * np.pi / (d * n)
    i = np.arange(n)
    return np.where(i <= n // 2, -i * dk, (n - i) * dk)


def inversion_image(S, R, dx, dy, dz):
    S = np.asarray(S, np.float64)
    R = np.asarray(R, np.float64)
    ny, nx, nz = S.shape
    kz = _k(nz, dz)[: nz // 2 + 1][None, None, :]
    kx = _k(nx, dx)[None, :, None]
    ky = (_k(ny, dy) if ny > 1 else np.zeros(1))[:, None, None]
    kk = np.sqrt(kx * kx + kz * kz + ky * ky)
    safe = np.where(kk > 1e-25, kk, 1.0)
    Sh, Rh = np.fft.rfftn(S), np.fft.rfftn(R)
    img = S * R
    for ka in (kz, kx, ky) if ny > 1 else (kz, kx):
        f = np.where(kk > 1e-25, 1j * ka / safe, 0.0)
        ds = np.fft.irfftn(f * Sh, s=S.shape, axes=(0, 1, 2))
        dr = np.fft.irfftn(f * Rh, s=S.shape, axes=(0, 1, 2))
        img = img - ds * dr
    return img
