"""CPU restatement of the trace time-dispersion / phase correction -
test infrastructure (the checker of the CUDA path, never the product).
PhaseCorrection (bgprtm/PhaseCorrection.cpp:14-235):

* constructor (:14-38): phase = phase_deg pi / 180, c_phase = exp(-i phase);
  tdsp_correction (global, default 2; 0 when do_tdsp is 0); with resampling
  (dtOut > 0, ntOut > 0) nt_dft = ntOut, dt_dft = dtOut, t_shift = t0Out - t0,
  else nt_dft = nt, dt_dft = dt, t_shift = 0, t0Out = t0; it_shift =
  int(t_shift / dt_dft), t_shift_frac = t_shift - it_shift dt_dft;
* init (:62-115): do_fft_dft = direction == BWD (or forced); the sin
  Jacobian for FWD; it0 = (do_fft_dft ? t0Out : t0) / dt_dft; dw = 2 pi /
  (ntfft dt); nw1 = min(nw, nearbyint(2 pi fmax / dw) + 1); per bin iw < nw1
  x = iw dw Dt, factor = 2 cos(x / 2) (Jacobian) or 2, dsp = (r acos-form +
  (1 - r) sin-form) dt_dft / Dt (0 without Dt or when skipped), and per output
  sample the phase phs (two forms, dt == dt_dft or not), T = exp(i phs) factor;
* fft_dft (:141-190) / dft_fft (:192-235): the transforms, the band's bins
  times c_phase * factor(w_pow) / ntfft, bin 0 real (halved before the table
  sum), the table sums or the inverse transform;
* applyForward / applyBackward (:116-140): the routing between them.

The table and the multipliers are float32 in the reference's operation order
(numpy float32 operations round like the C++ ones; the transcendental
functions may differ by an ulp); transforms and sums are float64.
libfftv (fft_r2c_fd, fft_c2r_bd, padfftv) is absent from the reference tree:
the forward transform is taken as unnormalised with exp(+i w t) and the
Nyquist bin packed into bin 0's imaginary part (every path clears it), the
backward one as the unnormalised Hermitian sum with exp(-i w t) - the only
conventions under which fft_dft with a dispersion-free table returns its
band-limited input.  Parity unpinned: PhaseCorrection.cpp does not compile as
it stands in the reference tree (a stray token after the constructor's
t_shift line and a repeated declaration of dsp in init) and libfftv is
missing, so the tests pin this restatement to closed-form answers instead."""
import math

import numpy as np

F32 = np.float32
FLT_PI = F32(np.pi)
FWD, BWD = 1, 2


def _nearbyint(v):
    return int(np.rint(v))


class Plan:
    """The constructor's and init()'s derived quantities."""

    def __init__(self, nt, dt, Dt, t0, fmax, direction, w_pow=0.0, phase_deg=0.0, do_tdsp=1, ntOut=-1, dtOut=-1.0,
                 t0Out=0.0, ntfft=None, tdsp_correction=2, skip_tdsp_correction=0, tdsp_acos_ratio=0.0,
                 skip_jacobian=False, transform=0):
        dt, Dt, t0, fmax = F32(dt), F32(Dt), F32(t0), F32(fmax)
        dtOut, t0Out = F32(dtOut), F32(t0Out)
        self.nt, self.ntfft, self.direction = nt, ntfft, direction
        self.nw = ntfft // 2 + 1
        self.phase = F32(F32(phase_deg) * FLT_PI) / F32(180)
        self.c_phase = np.complex64(complex(math.cos(-float(self.phase)), math.sin(-float(self.phase))))
        self.w_pow = F32(w_pow)
        skip = skip_tdsp_correction & direction
        self.tdsp = tdsp_correction if do_tdsp else 0
        self.resample = dtOut > 0 and ntOut > 0
        if self.resample:
            self.nt_dft, dt_dft, t_shift = ntOut, dtOut, F32(t0Out - t0)
        else:
            self.nt_dft, dt_dft, t_shift, t0Out = nt, dt, F32(0), t0
        it_shift = int(F32(t_shift / dt_dft))
        t_shift_frac = F32(t_shift - F32(F32(it_shift) * dt_dft))
        self.identity = not self.tdsp and self.w_pow == 0 and self.phase == 0
        self.do_fft_dft = direction == BWD
        if transform == 1:
            self.do_fft_dft = True
        elif transform == 2:
            self.do_fft_dft = False
        jac = direction == FWD and not skip and not skip_jacobian
        it0 = F32((t0Out if self.do_fft_dft else t0) / dt_dft)
        dw = 2.0 * math.pi / float(F32(F32(ntfft) * dt))
        self.nw1 = min(self.nw, _nearbyint(F32(float(F32(F32(2.0) * FLT_PI) * fmax) / dw)) + 1)
        nw1, nt_dft = self.nw1, self.nt_dft
        r = F32(tdsp_acos_ratio)
        self.table = None
        if self.tdsp:
            it = np.arange(nt_dft)
            T = np.zeros((nw1, nt_dft), np.complex64)
            for iw in range(nw1):
                x = float(iw) * dw * float(Dt)
                factor = F32(F32(2.0) * np.cos(F32(x / 2))) if jac else F32(2.0)
                if Dt == 0 or skip:
                    dsp = F32(0)
                else:
                    c = 1 - 0.5 * x * x  # outside [-1, 1] (w Dt > 2) C's acos gives NaN, and so does the table
                    acos_form = (math.acos(c) if -1.0 <= c <= 1.0 else math.nan) - x
                    sin_form = x - 2.0 * math.sin(x / 2.0)
                    dsp = F32((float(r) * acos_form + float(F32(1 - r)) * sin_form) * float(dt_dft) / float(Dt))
                lin = (it - it0).astype(F32) * dsp
                if dt == dt_dft:
                    wrap = np.fmod((it - it_shift).astype(np.int64) * iw, ntfft)  # C remainder
                    phs = (lin.astype(np.float64) - wrap * dw * float(dt_dft) +
                           float(F32(t_shift_frac * F32(iw))) * dw).astype(F32)
                else:
                    dwf = F32(dw)
                    b = (F32(dwf * dt_dft) * it.astype(F32)) * F32(iw)
                    c = F32(dwf * t_shift) * F32(iw)
                    phs = (lin - b + c).astype(F32)
                    n = np.rint(phs / F32(F32(2) * FLT_PI)).astype(np.int64)
                    phs = (phs - (n * 2).astype(F32) * FLT_PI).astype(F32)
                T[iw] = (np.cos(phs) * factor) + 1j * (np.sin(phs) * factor)
            self.table = T
        dwf = F32(2.0 * math.pi / float(F32(F32(ntfft) * dt)))
        scaler = F32(F32(1.0) / F32(ntfft))
        self.mul = np.zeros(nw1, np.complex64)
        for iw in range(nw1):
            f = F32(1) if self.w_pow == 0 else F32(0) if iw == 0 else F32(np.power(F32(F32(iw) * dwf), self.w_pow))
            self.mul[iw] = complex(F32(F32(self.c_phase.real * f) * scaler), F32(F32(self.c_phase.imag * f) * scaler))


def _forward(x, n):
    """libfftv::fft_r2c_fd as inferred: sum_t x_t exp(+i 2 pi k t / n), k <= n / 2."""
    return np.conj(np.fft.rfft(x.astype(np.float64), n=n, axis=-1))


def _inverse(X, n):
    """libfftv::fft_c2r_bd as inferred: the Hermitian sum of X_k exp(-i 2 pi k t / n)."""
    return np.fft.irfft(np.conj(X), n=n, axis=-1) * n


def _scale_band(p, X):
    X = X.copy()
    X[..., p.ntfft // 2] = 0  # the Nyquist bin (packed into bin 0 by libfftv)
    X[..., 0] = X[..., 0].real
    X[..., :p.nw1] *= p.mul.astype(np.complex128)
    X[..., 0] = X[..., 0].real
    return X


def fft_dft(p, x):
    """PhaseCorrection::fft_dft (:141-190) on traces [ntr][nt] -> [ntr][nt_dft]."""
    X = _scale_band(p, _forward(x, p.ntfft))
    if p.tdsp:
        Xb = X[..., :p.nw1].copy()
        Xb[..., 0] *= 0.5
        T = p.table.astype(np.complex128)
        return Xb.real @ T.real - Xb.imag @ T.imag
    y = _inverse(X, p.ntfft)
    if p.nt_dft > p.ntfft:
        raise ValueError("fft_dft without the table needs ntfft >= nt_dft")
    return y[..., :p.nt_dft]


def dft_fft(p, x):
    """PhaseCorrection::dft_fft (:192-235) on traces [ntr][nt] -> [ntr][nt]."""
    if p.resample:
        raise ValueError("dft_fft cannot resample")
    if p.tdsp:
        X = np.zeros(x.shape[:-1] + (p.nw,), np.complex128)
        X[..., :p.nw1] = x.astype(np.float64) @ np.conj(p.table.astype(np.complex128)).T
    else:
        X = _forward(x, p.ntfft)
    return _inverse(_scale_band(p, X), p.ntfft)[..., :p.nt]


def apply_forward(p, x):
    """PhaseCorrection::applyForward (:116-126)."""
    if p.direction != FWD:
        raise ValueError("applyForward needs direction FWD")
    if p.identity:
        return x.astype(np.float64)
    if p.resample:
        raise ValueError("applyForward cannot resample")
    if p.do_fft_dft and p.tdsp == 1:
        return fft_dft(p, x)
    return dft_fft(p, x)


def apply_backward(p, x, scaler=1.0, nt_out=-1):
    """PhaseCorrection::applyBackward (:128-140); scaler on the first nt_out
    samples of each output trace when nt_out > 0."""
    if p.identity:
        if p.resample:
            raise ValueError("the no-op cannot resample")
        return x.astype(np.float64)
    y = fft_dft(p, x) if (p.do_fft_dft or p.tdsp != 1) else dft_fft(p, x)
    if scaler != 1.0 and nt_out > 0:
        y = y.copy()
        y[..., :nt_out] *= float(F32(scaler))
    return y
