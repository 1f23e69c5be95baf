"""Pseudo-spectral engines on the GPU against the oracle: FFTWR2C
(FdEngine_r2c: cuFFT line transforms), FFTWR2R (FdEngine_r2r: cosine / sine
transform derivatives as line-matrix GEMMs), and the Derivative-path engines
FFTV and SINCOS on the same line operators - modelling traces of a VTI and a
TTI + Q shot, and an RTM image.  FP32 transforms against the oracle's
double sums: 1e-4, the engine's trace tolerance; images 1e-4 (atomic
receiver injection reorders sums).  Line lengths are even: for odd n the
FFTWR2C isign factor on bin n/2 gives its two passes a growing mode (the
operator steps with odd x, y and z run a few steps in the golden-fixture
tests)."""
import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200.propagator import Propagator, spread_coeffs
from konglong_b200.spec import ENGINE_FFTV, ENGINE_R2C, ENGINE_R2R, ENGINE_SINCOS, SNAP_FP32
from oracle import pyoracle as O
from tests.conftest import rel_l2
from tests.test_gpu_parity import _modelling, _rtm

pytestmark = pytest.mark.gpu


def _vti(nt, engine):
    shot = W.vti_cfd(scale=0.125, nt=nt)  # 64 x 64 x 50; the CFL bound (k1max = pi) is the same
    shot.spec.engine = engine
    return shot


SPECTRAL = [ENGINE_R2C, ENGINE_R2R, ENGINE_FFTV, ENGINE_SINCOS]


@pytest.mark.parametrize("engine", SPECTRAL)
@pytest.mark.parametrize("which", ["vti", "tti_q"])
def test_r2c_modelling_traces(which, engine):
    nts = 160
    shot = _vti(nts, engine) if which == "vti" else W.tti_q(scale=0.075, nt=nts, engine=engine)
    s = shot.spec
    assert s.pml3d  # requested, and ignored by the FFT engine on both sides
    q = W.q_coefficients(s.dt, shot.fpeak) if s.use_q else None
    g = Propagator(s)
    o = O.Oracle(s)
    if q:
        g.set_q_coeffs(*q)
        o.set_q_coeffs(*q)
    got = _modelling(shot, g, spread_coeffs, nts)
    want = _modelling(shot, o, spread_coeffs, nts)
    g.close()
    assert np.abs(want).max() > 0 and np.isfinite(got).all()
    assert rel_l2(got, want) < 1e-4


@pytest.mark.parametrize("engine", SPECTRAL)
def test_r2c_rtm_image(engine):
    nt = 120
    shot = _vti(nt, engine)
    g = Propagator(shot.spec)
    got = _rtm(shot, g, spread_coeffs, SNAP_FP32, nt, nt, shot.interval)
    g.close()
    want = _rtm(shot, O.Oracle(shot.spec), spread_coeffs, SNAP_FP32, nt, nt, shot.interval)
    assert np.abs(want).max() > 0
    assert rel_l2(got.reshape(want.shape), want) < 1e-4


@pytest.mark.parametrize("engine", SPECTRAL)
def test_pseudo_spectral_2d_grid(engine):
    """A 2-D grid (ny = 1: no y derivative, no y plans) through both engines:
    operator steps against the oracle."""
    from konglong_b200.spec import VTI, PropSpec
    nx, nz = 40, 36
    s = PropSpec(nx=nx, ny=1, nz=nz, dx=10.0, dy=10.0, dz=10.0, dt=0.0006, engine=engine, model_type=VTI,
                 nbnd=(6, 6, 0, 0, 6, 6), vmax=4500.0)
    rng = np.random.default_rng(4)
    model = dict(vel=(1800.0 + 2000.0 * rng.random(s.shape)).astype(np.float32),
                 eps=(0.2 * rng.random(s.shape)).astype(np.float32), dl=(0.08 * rng.random(s.shape)).astype(np.float32))
    w1 = rng.standard_normal(s.shape).astype(np.float32)
    out = []
    for cls in (Propagator, O.Oracle):
        x = cls(s)
        x.set_model(**model)
        x.put(0, np.zeros_like(w1))
        x.put(1, w1)
        for _ in range(3):
            x.kernel()
            x.update2nd()
            x.swap()
        out.append(np.asarray(x.get(1), np.float64).ravel())
    assert np.abs(out[1]).max() > 0
    assert rel_l2(out[0], out[1]) < 1e-5
