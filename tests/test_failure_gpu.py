"""Failure detection on the GPU, without faulting the GPU.

* Bounded device waits: a kernel waits on an mbarrier phase that nothing
  completes; the wait gives up after its poll limit, the host reads
  RTM_ERR_TIMEOUT, and the context stays usable (a shot run afterwards
  matches a fresh engine bit for bit).
* Non-finite wavefields: a NaN planted on the host, and a dt far above the
  stability bound, are both reported by the device scan; rtm_reset recovers.
"""
import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200._lib import STATUS_CODE, RtmError
from konglong_b200.propagator import Propagator, spread_coeffs
from konglong_b200.spec import FIELD_IMAGE, FIELD_W0, FIELD_W1

pytestmark = pytest.mark.gpu


def _shot(scale=0.25, nt=80):
    return W.iso128(scale=scale, nt=nt)


def _model_run(shot, p, nts):
    s = shot.spec
    p.set_model(**shot.model_arrays())
    k1, k2 = W.spread_band(s)
    src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    rcv = W.make_traceset(shot.rcv_pos[:16], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    p.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
    p.set_extraction(rcv, nts)
    p.reset()
    p.modelling(nts, -1, 1)
    return p.traces(), p.get(FIELD_W1)


def test_bounded_wait_times_out_and_context_survives():
    shot = _shot()
    p = Propagator(shot.spec)
    assert p.selftest_bounded_wait() == STATUS_CODE["RTM_ERR_TIMEOUT"]
    # the flag was consumed: a second self-test times out again, not earlier state
    assert p.selftest_bounded_wait() == STATUS_CODE["RTM_ERR_TIMEOUT"]
    tr, w1 = _model_run(shot, p, 60)
    q = Propagator(shot.spec)
    tr2, w12 = _model_run(shot, q, 60)
    np.testing.assert_array_equal(tr, tr2)
    np.testing.assert_array_equal(w1, w12)
    assert p.check_finite(FIELD_W1)


def test_planted_nan_is_detected_and_reset_recovers():
    shot = _shot()
    p = Propagator(shot.spec)
    p.set_model(**shot.model_arrays())
    p.reset()
    assert p.check_finite(FIELD_W0) and p.check_finite(FIELD_W1)
    with pytest.raises(RtmError) as e:  # no image before rtm_image_setup
        p.check_finite(FIELD_IMAGE)
    assert e.value.code == STATUS_CODE["RTM_ERR_ARG"]
    p.image_setup(0, 0, 1)
    assert p.check_finite(FIELD_IMAGE)
    w = np.zeros(shot.spec.shape, np.float32)
    w[3, 5, 7] = np.nan
    p.put(FIELD_W1, w)
    assert not p.check_finite(FIELD_W1)
    assert p.check_finite(FIELD_W0)
    p.kernel()  # the NaN spreads into w0 through the stencil
    assert not p.check_finite(FIELD_W0)
    p.reset()
    assert p.check_finite(FIELD_W0) and p.check_finite(FIELD_W1)


def test_unstable_dt_blows_up_and_is_detected():
    shot = _shot(nt=400)
    shot.spec.dt = 4.0 * shot.spec.dt  # far above the FD8 leapfrog bound
    p = Propagator(shot.spec)
    _model_run(shot, p, 400)
    assert not p.check_finite(FIELD_W1)
