"""Batched small shots: persistent launches per step over all shots (uneven
grids and step counts; ISO, VTI and TTI batches) must reproduce every shot's
own rtm_modelling."""
import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200._lib import STATUS_CODE, RtmError
from konglong_b200.propagator import Batch, Propagator, spread_coeffs
from konglong_b200.spec import FIELD_W0, FIELD_W1, TTI, VTI
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


def _tti(shots, seed=3):
    """The same shots with a tilted symmetry axis (TTI): smooth seeded tilt
    0-30 degrees and azimuth, the time step from the CFL rule."""
    rng = np.random.default_rng(seed)
    for sh in shots:
        s = sh.spec
        s.model_type = TTI
        theta = np.deg2rad(W.minmax(W.smooth_field(s.shape, 3.0, rng), 0.0, 30.0))
        phi = np.deg2rad(W.minmax(W.smooth_field(s.shape, 3.0, rng), 0.0, 360.0))
        sh.pjx = (-np.sin(theta) * np.cos(phi)).astype(np.float32)
        sh.pjy = (-np.sin(theta) * np.sin(phi)).astype(np.float32)
        s.dt = float(min(s.dt, W.cfl_dt(s, sh.vel, sh.eps, sh.dl, sh.pjx, sh.pjy)))
        sh.wavelet = W.ricker(sh.fpeak, s.dt, sh.nt)
    return shots


@pytest.mark.parametrize("model", ["vti", "tti"])
@pytest.mark.parametrize("tune", [False, True])
def test_anisotropic_batch_matches_per_shot(model, tune):
    """VTI / TTI shots of uneven grids and step counts through the batched
    gradient and divergence passes equal each shot's own rtm_modelling bit for
    bit (the batch runs the one-cell passes, which every FD8 anisotropic kernel
    equals), receivers to the warp-sum rounding."""
    shots = W.small_shots(nshots=5, seed=11, size=(36, 72), steps=(40, 100), nrec=6, model=VTI)
    if model == "tti":
        shots = _tti(shots)
    nts = [sh.nt for sh in shots]
    ref = []
    for sh in shots:
        p = _setup(sh)
        p.modelling(sh.nt, -1, 1)
        ref.append((p.traces(), p.get(FIELD_W1), p.get(FIELD_W0)))
        p.close()
    assert all(np.isfinite(r[1]).all() and np.abs(r[1]).max() > 0 for r in ref)
    ps = [_setup(sh) for sh in shots]
    b = Batch(ps)
    if tune:
        b.autotune(3)
        for p in ps:
            p.reset()
    b.modelling(nts, -1, 1)
    for (tr, w1, w0), p in zip(ref, ps):
        np.testing.assert_array_equal(p.get(FIELD_W1), w1)
        np.testing.assert_array_equal(p.get(FIELD_W0), w0)
        assert rel_l2(p.traces(), tr) < 1e-5
    b.close()


def test_batch_rejects_mixed_model_types():
    iso = W.small_shots(nshots=1, seed=1, size=(36, 40), steps=(10, 10), nrec=2)[0]
    vti = W.small_shots(nshots=1, seed=2, size=(36, 40), steps=(10, 10), nrec=2, model=VTI)[0]
    ps = [_setup(iso), _setup(vti)]
    with pytest.raises(RtmError) as e:
        Batch(ps)
    assert e.value.code == STATUS_CODE["RTM_ERR_UNSUPPORTED"]
