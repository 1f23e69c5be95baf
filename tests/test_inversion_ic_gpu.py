"""INVERSION imaging condition on the GPU (cuFFT k-domain derivatives): one
imaging term against the float64 restatement, and the loop driver's backward
pass against the same pass driven by stepwise calls."""
import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200.spec import BACKWARD, FIELD_IMAGE, FIELD_W0, FORWARD, IC_IMAGE1, IC_INVERSION, SNAP_FP32
from oracle import ic_oracle as IC
from tests.conftest import rel_l2
from tests.test_iso_variants_gpu import _engine, _iso_shot

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("grid", [(40, 24, 48), (37, 20, 43)])
def test_inversion_term_matches_oracle(grid):
    shot = _iso_shot(*grid, nt=10)
    s = shot.spec
    p, _, _ = _engine(shot, 0)
    rng = np.random.default_rng(9)
    A = W.smooth_field(s.shape, 2.0, rng).astype(np.float32)
    B = W.smooth_field(s.shape, 1.5, rng).astype(np.float32)
    p.snapshot_setup(SNAP_FP32, 1)
    p.put(FIELD_W0, A)
    p.snapshot_store(0)
    p.put(FIELD_W0, B)
    p.image_setup(0, 0, 0)  # no tapers: the terms act on A and B themselves
    p.image_condition(IC_INVERSION)
    p.image_accumulate(0)
    got = p.get(FIELD_IMAGE).reshape(s.shape)
    want = IC.inversion_image(A, B, s.dx, s.dy, s.dz)
    assert np.abs(want).max() > 0
    assert rel_l2(got, want) < 1e-5
    assert rel_l2(got, A * B) > 1e-2  # the derivative terms are not negligible
    p.close()


def test_loop_inversion_equals_stepwise_calls():
    shot = _iso_shot(40, 24, 48, nt=60)
    s, nt, iv = shot.spec, shot.nt, shot.interval
    nslots = (nt - 1) // iv + 1
    rng = np.random.default_rng(5)
    images = []
    for stepwise in (False, True):
        p, src, rcv = _engine(shot, 0)
        data = (rng.standard_normal((rcv.ntr, nt)) * 1e3).astype(np.float32) if not images else data
        p.snapshot_setup(SNAP_FP32, nslots)
        p.reset()
        p.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
        p.migration(FORWARD, 0, nt, -1, iv)
        p.reset()
        p.image_setup(3, 4, 1)
        p.image_condition(IC_INVERSION)
        p.set_injection(rcv, data, s.dt_dxyz)
        if not stepwise:
            p.migration(BACKWARD, nt - 1, -1, -1, iv)
        else:  # the loop's order: step, inject sample it+1, imaging term on this step's field, swap
            for it in range(nt - 1, -1, -1):
                p.kernel()
                p.update2nd()
                p.inject(it + 1)
                if it % iv == 0:
                    p.image_accumulate(it // iv)
                p.swap()
        images.append(p.get(FIELD_IMAGE))
        p.close()
    assert np.isfinite(images[0]).all() and np.abs(images[0]).max() > 0
    assert rel_l2(images[1], images[0]) < 1e-5
