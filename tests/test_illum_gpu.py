"""Source illumination and shot illumination compensation on the GPU: the
illumination the fused imaging condition accumulates equals the sum of the
squared source snapshots (trivial tapers), and the compensation (box smoothing,
damping factor, edge tapers, image scaling) matches the CPU restatement."""
import numpy as np
import pytest

from konglong_b200.spec import BACKWARD, FIELD_ILLUM, FIELD_IMAGE, FORWARD, SNAP_FP32
from oracle import illum_oracle as IO
from tests.conftest import rel_l2
from tests.test_iso_variants_gpu import _engine, _iso_shot

pytestmark = pytest.mark.gpu


def _rtm_with_illum(shot, p, src, rcv):
    nt = shot.nt
    nslots = (nt - 1) // shot.interval + 1
    p.snapshot_setup(SNAP_FP32, nslots)
    p.reset()
    p.set_injection(src, shot.wavelet[None, :], shot.spec.dt_dxyz)
    p.migration(FORWARD, 0, nt, -1, shot.interval)
    rng = np.random.default_rng(5)
    data = (rng.standard_normal((rcv.ntr, nt)) * 1e3).astype(np.float32)
    p.reset()
    p.image_setup(0, 0, 1)  # no time / depth taper: the source term is the decoded snapshot
    p.illum_setup(True)
    p.set_injection(rcv, data, shot.spec.dt_dxyz)
    p.migration(BACKWARD, nt - 1, -1, -1, shot.interval)
    return nslots


@pytest.mark.parametrize("grid", [(40, 24, 48), (37, 20, 42)])  # 4-cell and one-cell imaging paths
def test_illumination_and_compensation(grid):
    shot = _iso_shot(*grid, nt=120)
    p, src, rcv = _engine(shot, 0)
    nslots = _rtm_with_illum(shot, p, src, rcv)
    illum = p.get(FIELD_ILLUM)
    want = np.zeros_like(illum)
    for s in range(nslots - 1, -1, -1):  # the backward loop's order
        w = p.snapshot_load(s)
        want = (want + w * w).astype(np.float32)
    assert want.max() > 0
    assert rel_l2(illum, want) < 1e-5
    image = p.get(FIELD_IMAGE)
    f_ref, img_ref = IO.compensate(illum.reshape(shot.spec.shape), image.reshape(shot.spec.shape))
    p.illum_compensate()
    assert rel_l2(p.get(FIELD_ILLUM), f_ref) < 1e-5
    assert rel_l2(p.get(FIELD_IMAGE), img_ref) < 1e-5
    p.close()

