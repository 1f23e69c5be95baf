"""The CPU restatement of the illumination smoothing (oracle/illum_oracle.py)
against a direct windowed mean with the reference's edge rule."""
import numpy as np

from oracle import illum_oracle as IO


def test_box_average_restatement():
    """The restated running average equals a direct windowed mean with replicated edges."""
    rng = np.random.default_rng(3)
    a = rng.random((30, 5)).astype(np.float32)
    h = 4
    pad = np.concatenate([np.repeat(a[:1], h + 1, 0), a, np.repeat(a[-1:], h, 0)])
    # the reference drops a[k-h-1] (clamped to index 0) and adds a[k+h] (clamped to the end)
    direct = np.array([pad[k + 1:k + 2 * h + 2].mean(0) for k in range(30)])
    assert np.allclose(IO.avg1d(a, h), direct, rtol=1e-5, atol=1e-6)


def test_smoothing_matches_compiled_reference(golden):
    """The restated avgVolume3D / avgVolume2D against the reference's own
    volumefilter.cpp (oracle/_ref; its -ffast-math build may reassociate the
    running sums: 2e-6)."""
    from tests.golden_inputs import ILLUM_SMOOTH, illum_input
    for name, (shape, hxy, hz) in ILLUM_SMOOTH.items():
        ref = golden[f"illum_smooth_{name}"]
        got = IO.smooth(illum_input(name), hxy, hz)
        assert np.abs(got - ref).max() <= 2e-6 * np.abs(ref).max(), name
