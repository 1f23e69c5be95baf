"""Batched small shots: one persistent launch per step over all shots (uneven
grids and step counts) must reproduce every shot's own rtm_modelling."""
import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200._lib import STATUS_CODE, RtmError
from konglong_b200.propagator import Batch, Propagator, spread_coeffs
from konglong_b200.spec import FIELD_W0, FIELD_W1
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _setup(shot):
    s = shot.spec
    p = Propagator(s)
    p.set_model(**shot.model_arrays())
    k1, k2 = W.spread_band(s)
    src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    rcv = W.make_traceset(shot.rcv_pos, s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    p.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
    p.set_extraction(rcv, shot.nt)
    p.reset()
    return p


@pytest.mark.parametrize("tune", [False, True])
def test_batch_matches_per_shot(tune):
    shots = W.small_shots(nshots=6, seed=7, size=(36, 72), steps=(40, 110), nrec=6)
    nts = [sh.nt for sh in shots]
    ref = []
    for sh in shots:
        p = _setup(sh)
        p.modelling(sh.nt, -1, 1)
        ref.append((p.traces(), p.get(FIELD_W1), p.get(FIELD_W0)))
        p.close()
    ps = [_setup(sh) for sh in shots]
    b = Batch(ps)
    if tune:
        b.autotune(3)
        for p in ps:
            p.reset()
    b.modelling(nts, -1, 1)
    assert b.last_ms > 0
    for (tr, w1, w0), p in zip(ref, ps):
        # stencil, injection and swap parity are the same arithmetic: equal fields
        np.testing.assert_array_equal(p.get(FIELD_W1), w1)
        np.testing.assert_array_equal(p.get(FIELD_W0), w0)
        # receivers: a warp sum per receiver vs the handle's grouped gather
        assert rel_l2(p.traces(), tr) < 1e-5
    b.close()


def test_batch_rejects_unsupported_shots():
    shot = W.vti_cfd(scale=0.08, nt=10)
    p = Propagator(shot.spec)
    p.set_model(**shot.model_arrays())
    with pytest.raises(RtmError) as e:
        Batch([p])
    assert e.value.code == STATUS_CODE["RTM_ERR_UNSUPPORTED"]
