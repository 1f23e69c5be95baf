"""Snapshot offload (the reference's CacheFile / AsyncIO spill, restated as pinned
host slots with device staging slots): the slots the forward loop copies to the
host decode to the same volumes as device-resident slots, and an RTM shot with
offloaded snapshots gives the image of the device-resident run - FP32, COMPRESS_16
and FP16 slots, 2 and 3 staging slots, a loop longer than one 256-step graph."""
import numpy as np
import pytest

from konglong_b200._lib import STATUS_CODE, RtmError
from konglong_b200.spec import BACKWARD, FIELD_IMAGE, FORWARD, SNAP_AE, SNAP_C16, SNAP_FP16S, SNAP_FP32
from tests.conftest import rel_l2
from tests.test_iso_variants_gpu import _engine, _iso_shot

pytestmark = pytest.mark.gpu


def _forward(shot, p, src, fmt, nstage):
    nt = shot.nt
    nslots = (nt - 1) // shot.interval + 1
    p.snapshot_setup(fmt, nslots)
    if nstage:
        p.snapshot_offload(nstage)
    p.reset()
    p.set_injection(src, shot.wavelet[None, :], shot.spec.dt_dxyz)
    p.migration(FORWARD, 0, nt, -1, shot.interval)
    return nslots


def _backward(shot, p, rcv):
    nt = shot.nt
    rng = np.random.default_rng(5)
    data = (rng.standard_normal((rcv.ntr, nt)) * 1e3).astype(np.float32)
    p.reset()
    p.image_setup(3, 4, 1)
    p.set_injection(rcv, data, shot.spec.dt_dxyz)
    p.migration(BACKWARD, nt - 1, -1, -1, shot.interval)
    return p.get(FIELD_IMAGE)


@pytest.mark.parametrize("fmt,nstage", [(SNAP_FP32, 2), (SNAP_C16, 3), (SNAP_FP16S, 2)])
def test_offloaded_rtm_equals_device_slots(fmt, nstage):
    shot = _iso_shot(40, 24, 48, nt=300)  # 300 steps: two CUDA-graph chunks
    ref, src, rcv = _engine(shot, 0)
    nslots = _forward(shot, ref, src, fmt, 0)
    off, _, _ = _engine(shot, 0)
    assert _forward(shot, off, src, fmt, nstage) == nslots
    for slot in (0, 1, nslots // 2, nslots - 1):
        np.testing.assert_array_equal(off.snapshot_load(slot), ref.snapshot_load(slot))
    img_ref, img_off = _backward(shot, ref, rcv), _backward(shot, off, rcv)
    assert np.abs(img_ref).max() > 0
    # receiver injection uses atomic adds, whose order varies between runs
    assert rel_l2(img_off, img_ref) < 1e-5
    # a second backward pass reuses the staged slots and the host copies
    assert rel_l2(_backward(shot, off, rcv), img_off) < 1e-5
    ref.close(), off.close()


def test_offload_arguments():
    shot = _iso_shot(40, 24, 48, nt=20)
    p, _, _ = _engine(shot, 0)
    p.snapshot_setup(SNAP_FP32, 3)
    for bad in (1, 9, -1):
        with pytest.raises(RtmError) as e:
            p.snapshot_offload(bad)
        assert e.value.code == STATUS_CODE["RTM_ERR_ARG"]
    p.snapshot_offload(2)
    p.snapshot_offload(0)  # back to device slots
    p.close()
