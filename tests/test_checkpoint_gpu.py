"""Store / recompute: checkpoints of the propagation state and the checkpointed
RTM shot.  Loading a checkpoint and running the loop again reproduces the
wavefields bit for bit (FD8 TTI + Q with FP32 and BF16 Q memory, compact-FD
VTI, ISO FD8, FP16 state), and an RTM shot whose snapshots are recomputed one
segment at a time gives the image of the shot that stores them all (to 1e-5:
the backward receiver injection uses atomic adds)."""
import dataclasses

import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200.propagator import Propagator, checkpoint_plan, spread_coeffs
from konglong_b200.spec import FIELD_W0, FIELD_W1, FORWARD, SNAP_C16, SNAP_FP16S, SNAP_FP32, TTI, VTI
from tests.conftest import rel_l2
from tests.test_aniso_variants_gpu import _aniso_shot

pytestmark = pytest.mark.gpu


def _setup(shot):
    s = shot.spec
    p = Propagator(s)
    if s.use_q:
        p.set_q_coeffs(*W.q_coefficients(s.dt, shot.fpeak))
    p.set_model(**shot.model_arrays())
    k1, k2 = W.spread_band(s)
    src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    rcv = W.make_traceset(shot.rcv_pos, s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    return p, src, rcv


def _shots():
    tq = _aniso_shot(45, 26, 56, TTI, use_q=True, nt=90)
    tqb = _aniso_shot(45, 26, 56, TTI, use_q=True, nt=90)
    tqb.spec = dataclasses.replace(tqb.spec, q_bf16=True)
    vcfd = W.vti_cfd(scale=0.1, nt=90)
    iso = W.iso128(scale=0.3, nt=90)
    f16 = _aniso_shot(40, 22, 48, VTI, nt=90)
    f16.spec = dataclasses.replace(f16.spec, state_fp16=True)
    return {"tti_q": tq, "tti_q_bf16": tqb, "vti_cfd": vcfd, "iso": iso, "vti_fp16_state": f16}


@pytest.mark.parametrize("name", ["tti_q", "tti_q_bf16", "vti_cfd", "iso", "vti_fp16_state"])
def test_checkpoint_reproduces_the_loop(name):
    shot = _shots()[name]
    p, src, _ = _setup(shot)
    nb = p.checkpoint_setup(2)
    assert nb >= 2 * 4 * shot.spec.n // (2 if shot.spec.state_fp16 else 1)
    p.reset()
    p.set_injection(src, shot.wavelet[None, :], shot.spec.dt_dxyz)
    p.migration(FORWARD, 0, 40, -1, 1000)
    p.checkpoint_save(1)
    p.migration(FORWARD, 40, 75, -1, 1000)
    want = p.get(FIELD_W0), p.get(FIELD_W1)
    assert np.abs(want[0]).max() > 0
    p.migration(FORWARD, 75, 90, -1, 1000)  # move on, then go back
    p.checkpoint_load(1)
    p.migration(FORWARD, 40, 75, -1, 1000)
    got = p.get(FIELD_W0), p.get(FIELD_W1)
    for a, b in zip(want, got):
        np.testing.assert_array_equal(a, b)
    p.close()


@pytest.mark.parametrize("name,fmt,seg_slots", [("tti_q", SNAP_FP32, 5), ("tti_q_bf16", SNAP_FP16S, 7),
                                                ("vti_cfd", SNAP_C16, 4), ("iso", SNAP_FP32, 23)])
def test_checkpointed_rtm_equals_stored(name, fmt, seg_slots):
    shot = _shots()[name]
    nt, interval = shot.nt, 4
    p, src, rcv = _setup(shot)
    data = (np.random.default_rng(5).standard_normal((rcv.ntr, nt)) * 1e3).astype(np.float32)
    ref = p.rtm_shot(src, shot.wavelet[None, :], rcv, data, nt, nt, interval, snap_fmt=fmt, ntaper_t=3,
                     ntaper_z=4)[0]
    img, ms = p.rtm_shot_checkpointed(src, shot.wavelet[None, :], rcv, data, nt, nt, interval, seg_slots,
                                      snap_fmt=fmt, ntaper_t=3, ntaper_z=4)
    nseg = len(checkpoint_plan(nt, interval, seg_slots))
    assert np.abs(ref).max() > 0
    assert (ms["recompute"] > 0) == (nseg > 1)
    assert rel_l2(img, ref) < 1e-5, f"{nseg} segments"
    p.close()
