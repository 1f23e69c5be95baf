"""Double-grid IMAGE1 imaging condition on the GPU: one imaging term and the
illumination on the doubled grid against the float64 restatement, the loop
driver's backward pass against the same pass driven by stepwise calls, and the
factor combinations the C ABI refuses."""
import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200._lib import RtmError
from konglong_b200.spec import BACKWARD, FIELD_W0, FORWARD, IC_INVERSION, SNAP_FP32
from oracle import ic_double_oracle as D
from tests.conftest import rel_l2
from tests.test_iso_variants_gpu import _engine, _iso_shot

pytestmark = pytest.mark.gpu


def _shot(grid, nt):
    shot = _iso_shot(*grid, nt=nt)
    if grid[1] == 1:
        shot.spec.nbnd = (6, 6, 0, 0, 6, 6)
    return shot


# even and odd line lengths (the Nyquist bin of the half shift), 3-D and 2-D grids
@pytest.mark.parametrize("grid,dbl", [((40, 24, 48), (2, 2, 2)), ((37, 21, 43), (2, 2, 2)),
                                      ((48, 1, 40), (2, 2, 1)), ((45, 1, 39), (2, 1, 1))])
def test_double_grid_term_matches_oracle(grid, dbl):
    shot = _shot(grid, 10)
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
    p.illum_setup(True)
    p.image_double(*dbl)
    p.image_accumulate(0)
    got = p.get_image_double()
    cubes, s0 = D.image_step(A.reshape(s.shape), B.reshape(s.shape), *dbl)
    want = D.interleave(cubes, *dbl)
    assert got.shape == want.shape and np.abs(want).max() > 0
    assert rel_l2(got, want) < 2e-5, rel_l2(got, want)
    # the half-shifted copies are not copy 0
    assert rel_l2(got, D.interleave([cubes[0]] * len(cubes), *dbl)) > 1e-2
    il = p.get_illum_double()
    want_il = D.interp_illum((s0 * s0).astype(np.float32), *dbl)
    assert rel_l2(il, want_il) < 2e-5, rel_l2(il, want_il)
    p.close()


def test_loop_double_grid_equals_stepwise_calls():
    shot = _shot((40, 24, 48), 60)
    s, nt, iv = shot.spec, shot.nt, shot.interval
    nslots = (nt - 1) // iv + 1
    rng = np.random.default_rng(5)
    data = (rng.standard_normal((15, nt)) * 1e3).astype(np.float32)
    images = []
    for stepwise in (False, True):
        p, src, rcv = _engine(shot, 0)
        p.snapshot_setup(SNAP_FP32, nslots)
        p.reset()
        p.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
        p.migration(FORWARD, 0, nt, -1, iv)
        p.reset()
        p.image_setup(3, 4, 1)
        p.image_double(2, 2, 2)
        p.set_injection(rcv, data[:rcv.ntr], s.dt_dxyz)
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
        images.append(p.get_image_double())
        p.close()
    assert np.isfinite(images[0]).all() and np.abs(images[0]).max() > 0
    assert rel_l2(images[1], images[0]) < 1e-5


def test_refused_factor_combinations():
    p, _, _ = _engine(_shot((40, 24, 48), 10), 0)
    for dbl in [(2, 2, 1), (2, 1, 2), (2, 1, 1), (1, 2, 2), (3, 2, 2)]:
        with pytest.raises(RtmError):
            p.image_double(*dbl)
    p.image_double(1, 1, 1)  # off: accepted
    p.image_condition(IC_INVERSION)
    with pytest.raises(RtmError):
        p.image_double(2, 2, 2)
    p.close()
