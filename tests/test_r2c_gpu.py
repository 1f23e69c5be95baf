"""FFTWR2C engine (pseudo-spectral first derivatives, FdEngine_r2c) on the
GPU against the oracle: modelling traces of a VTI and a TTI + Q shot, and an
RTM image.  cuFFT transforms in FP32 against the oracle's circulant in
double: 1e-4, the engine's trace tolerance; images 1e-4 (atomic receiver
injection reorders sums).  Line lengths are even: for odd n the reference's
isign factor on bin n/2 gives the two passes a growing mode (the operator
steps with odd x, y and z run a few steps in the golden-fixture tests)."""
import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200.propagator import Propagator, spread_coeffs
from konglong_b200.spec import ENGINE_R2C, SNAP_FP32
from oracle import pyoracle as O
from tests.conftest import rel_l2
from tests.test_gpu_parity import _modelling, _rtm

pytestmark = pytest.mark.gpu


def _vti(nt):
    shot = W.vti_cfd(scale=0.125, nt=nt)  # 64 x 64 x 50; the CFL bound (k1max = pi) is the same
    shot.spec.engine = ENGINE_R2C
    return shot


@pytest.mark.parametrize("which", ["vti", "tti_q"])
def test_r2c_modelling_traces(which):
    nts = 160
    shot = _vti(nts) if which == "vti" else W.tti_q(scale=0.075, nt=nts, engine=ENGINE_R2C)
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


def test_r2c_rtm_image():
    nt = 120
    shot = _vti(nt)
    g = Propagator(shot.spec)
    got = _rtm(shot, g, spread_coeffs, SNAP_FP32, nt, nt, shot.interval)
    g.close()
    want = _rtm(shot, O.Oracle(shot.spec), spread_coeffs, SNAP_FP32, nt, nt, shot.interval)
    assert np.abs(want).max() > 0
    assert rel_l2(got.reshape(want.shape), want) < 1e-4
