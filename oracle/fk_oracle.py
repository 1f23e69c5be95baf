"""CPU restatement of the receiver FK true-amplitude / deghost spreading in
the space domain - test infrastructure (the checker of the CUDA path, never
the product).  Receiver::spread_sdomain (bgprtm/Receiver.cpp:851-1010), the
default of Receiver::spread (fk_domain SDOMAIN, :1012-1041):

* every trace is spread onto the (ny, nx) receiver grid with its separable x / y
  kernels (Receiver::spreadCoeffs :306-363, apply_src_coefxy :509-530:
  wf += (trace * kx) * ky), zero-padded to ntfft samples;
* forward real FFT over (y, x, t), unnormalised;
* per bin: ky / kx = get_wavenumber (:605-617), k = iw * dwv,
  tmp = 1 - (kx^2 + ky^2) / k^2; evanescent bins (tmp <= 0) and DC are zeroed;
  factor = (trueamp ? sqrt(tmp) : 1) * scalar, scalar = sqrt(1 / (nkx nky ntfft));
  deghost: kzdz = k sqrt(tmp) z, factor *= (kzdz >= pi/2 ? 1 : sin(kzdz) <= thr ?
  1/thr : 1/sin(kzdz)) * 0.5, the low-cut ramp on bins iw <= iw_lp, and the bin is
  multiplied by i * factor * side; otherwise by factor;
* inverse real FFT, unnormalised; the first nt samples of each column.

The per-bin arithmetic is float32 in the reference's order (numpy float32
operations round like the C++ ones).  With deghost, the product on the
Nyquist frequency plane (even ntfft) is anti-Hermitian in (ky, kx); an inverse
real FFT reads only part of it and FFTW and cuFFT need not read the same part,
so that plane is zeroed here and in the engine (band-limited data carry
nothing there).  libfftv::padfftv, which chooses ntfft, is absent: ntfft is an
input.  Parity: restated from the reference's source (Receiver.cpp needs
yaml-cpp, FFTW and libCommon to build), unpinned against compiled code."""
import numpy as np

from oracle import pyoracle as O

F32 = np.float32


def wavenumbers(n, dk):
    """Receiver::get_wavenumber: i dk up to n/2, then (i - n) dk (float)."""
    if n == 1:
        return np.zeros(1, F32)
    i = np.arange(n)
    return np.where(i < n // 2 + 1, i, i - n).astype(F32) * F32(dk)


def spread_grid(nx, ny, nt, ntfft, xy, traces, khpass, khcut, nlimit, ntaper=10):
    g = np.zeros((ny, nx, ntfft), F32)
    for r in range(len(traces)):
        ox, kx = O.spread_coeffs(nx, float(xy[r][0]), khpass, khcut, nlimit if nx > 1 else 1, False,
                                 ntaper if nx > 1 else 0)
        oy, ky = O.spread_coeffs(ny, float(xy[r][1]), khpass, khcut, nlimit if ny > 1 else 1, False,
                                 ntaper if ny > 1 else 0)
        tr = np.asarray(traces[r], F32)[:nt]
        for j in range(len(ky)):
            for i in range(len(kx)):
                g[oy + j, ox + i, :nt] += (tr * kx[i]) * ky[j]
    return g


def fk_filter(spec, nx, ny, ntfft, dt, dx, dy, vsurf, z, trueamp, deghost, side, flcut, flpass, thr, scalar=None):
    """The per-bin product on the half spectrum [ny][nx][nw]; `scalar` is
    spread_sdomain's sqrt(1 / (nx ny ntfft)) unless given (spread_kdomain: 1)."""
    nw = ntfft // 2 + 1
    dkx = F32(0.0) if nx == 1 else F32(2.0 * np.pi / np.float64(F32(dx) * F32(nx)))
    dky = F32(0.0) if ny == 1 else F32(2.0 * np.pi / np.float64(F32(dy) * F32(ny)))
    dwv = F32(2.0 * np.pi / np.float64(F32(F32(dt) * F32(ntfft)) * F32(vsurf)))
    kx, ky = wavenumbers(nx, dkx), wavenumbers(ny, dky)
    kw = np.arange(nw).astype(F32) * dwv
    scalar = F32(np.sqrt(1.0 / nx / ny / ntfft)) if scalar is None else F32(scalar)
    iw_lc = int(np.rint(F32(F32(F32(flcut) * F32(dt)) * F32(ntfft))))
    iw_lp = int(np.rint(F32(F32(F32(flpass) * F32(dt)) * F32(ntfft))))
    out = np.zeros_like(spec)
    kh2 = (kx[None, :] * kx[None, :] + ky[:, None] * ky[:, None]).astype(F32)  # [ny][nx]
    for iw in range(1, nw):
        k = kw[iw]
        tmp = (F32(1.0) - kh2 / (k * k)).astype(F32)
        live = tmp > 0
        cosv = np.sqrt(np.where(live, tmp, F32(0))).astype(F32)
        f = (cosv if trueamp else np.ones_like(cosv)) * scalar
        f = f.astype(F32)
        if deghost:
            if ntfft % 2 == 0 and iw == nw - 1:
                continue  # the Nyquist plane (see the module note)
            kzdz = ((k * cosv).astype(F32) * F32(z)).astype(F32)
            sinv = np.sin(kzdz).astype(F32)
            g = np.where(kzdz >= F32(np.pi / 2), F32(1), np.where(sinv <= F32(thr), F32(1) / F32(thr),
                                                                   F32(1) / np.where(sinv > 0, sinv, F32(1))))
            f = (f * g.astype(F32)).astype(F32) * F32(0.5)
            if iw <= iw_lc:
                f = f * F32(0)
            elif iw <= iw_lp:
                f = f * (F32(0.5) * (F32(1) - F32(np.cos(F32(np.pi) * F32(iw - iw_lc) / F32(iw_lp - iw_lc + 1)))))
            out[:, :, iw] = np.where(live, spec[:, :, iw] * (1j * f * side), 0)
        else:
            out[:, :, iw] = np.where(live, spec[:, :, iw] * f, 0)
    return out


def fk_deghost(nx, ny, nt, ntfft, dt, dx, dy, xy, traces, vsurf, z, trueamp, deghost, side=-1,
               flcut=0.0, flpass=0.0, thr=0.1, khpass=0.4, khcut=0.48, nlimit=20):
    """Receiver grid traces [ny][nx][nt] (float64) after spread_sdomain."""
    g = spread_grid(nx, ny, nt, ntfft, xy, traces, khpass, khcut, nlimit).astype(np.float64)
    spec = np.fft.rfftn(g, axes=(0, 1, 2))
    spec = fk_filter(spec, nx, ny, ntfft, dt, dx, dy, vsurf, z, trueamp, deghost, side, flcut, flpass, thr)
    out = np.fft.irfftn(spec, s=(ny, nx, ntfft), axes=(0, 1, 2)) * (nx * ny * ntfft)
    return out[:, :, :nt]


def ktaper(n, k, k1, k2):
    """Receiver::get_ktaper (bgprtm/Receiver.cpp:619-639): 1 below 2 k1 kmax,
    0 above 2 k2 kmax, cos^2 between (float)."""
    kmax = abs(F32(k[n // 2]))
    a, b = F32(kmax * F32(k1 * 2)), F32(kmax * F32(k2 * 2))
    ak = np.abs(k).astype(F32)
    t = np.cos((ak - a) / (b - a) * np.pi / 2.0) ** 2
    return np.where(ak < a, F32(1), np.where(ak > b, F32(0), t)).astype(F32)


def fk_deghost_kdomain(nx, ny, nt, ntfft, dt, dx, dy, xy_m, traces, vsurf, z, trueamp, deghost, side=-1,
                       flcut=0.0, flpass=0.0, thr=0.1, fmax=60.0, khpass=0.4, khcut=0.48):
    """Receiver::spread_kdomain (bgprtm/Receiver.cpp:641-849): each trace,
    scaled by sqrt(1 / (nx ny ntfft)), is transformed in time and summed into
    the (ky, kx) grid with the phase shifts exp(-i (kx x + ky y)) of its offsets
    from the grid origin and the k tapers; the per-bin product is
    spread_sdomain's without the scalar, with the ghost threshold scaled by
    sin(2 pi fmax z / vsurf) when that angle is below pi / 2 (:792-794); then
    the inverse FFT over (y, x, t).  nx > 1 (with nx = 1 the reference's x taper
    is 0 / 0)."""
    nw = ntfft // 2 + 1
    dkx = F32(2.0 * np.pi / np.float64(F32(dx) * F32(nx)))
    dky = F32(0.0) if ny == 1 else F32(2.0 * np.pi / np.float64(F32(dy) * F32(ny)))
    kx, ky = wavenumbers(nx, dkx), wavenumbers(ny, dky)
    tkx = ktaper(nx, kx, khpass, khcut)
    tky = ktaper(ny, ky, khpass, khcut) if ny > 1 else np.ones(1, F32)
    scalar = F32(np.sqrt(1.0 / nx / ny / ntfft))
    tw = np.zeros((len(traces), ntfft), np.float64)
    tw[:, :nt] = (np.asarray(traces, F32)[:, :nt] * scalar).astype(F32)
    T = np.fft.rfft(tw, axis=1)                                   # [nr][nw]
    xy_m = np.asarray(xy_m, F32)
    sx = np.exp(-1j * (xy_m[:, 0:1] * kx[None, :]).astype(F32)) * tkx[None, :]      # [nr][nx]
    sy = np.exp(-1j * (xy_m[:, 1:2] * ky[None, :]).astype(F32)) * tky[None, :]      # [nr][ny]
    spec = np.einsum("ry,rx,rw->yxw", sy, sx, T)
    thr_eff = F32(thr)
    kzdzmax = F32(F32(F32(F32(fmax) * F32(2 * np.pi)) / F32(vsurf)) * F32(z))
    if kzdzmax < F32(np.pi / 2):
        thr_eff = F32(thr_eff * np.sin(kzdzmax))
    spec = fk_filter(spec, nx, ny, ntfft, dt, dx, dy, vsurf, z, trueamp, deghost, side, flcut, flpass, thr_eff,
                     scalar=F32(1))
    out = np.fft.irfftn(spec, s=(ny, nx, ntfft), axes=(0, 1, 2)) * (nx * ny * ntfft)
    return out[:, :, :nt]
