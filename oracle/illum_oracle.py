"""CPU restatement of the shot illumination compensation - test infrastructure
(the checker of the CUDA path, never the product):

* avgVolume1D / avgVolume3D / avgVolume2D (bgprtm/volumefilter.cpp:59-135): running
  box averages with the reference's edge rule (the first value counted h+1 times) and
  its order of float32 operations (one add and one subtract per step);
* ImagingCondition::computeDamping / applyDamping (bgprtm/ImagingCondition.cpp:600-689):
  mean in float64, factor 1 / (avg (a + w e^-a)), 10-cell x / y cosine edge tapers,
  image *= factor.

Volumes are numpy arrays of shape (ny, nx, nz) (z fastest, the reference layout).
Parity: the box averages are pinned against the reference's own volumefilter.cpp
(compiled into oracle/_ref with a stand-in for libFFTV's transpose; fixtures in
tests/golden, agreement 1e-6 under the reference build's -ffast-math);
computeDamping / applyDamping are restated (ImagingCondition.cpp needs libFFTV's
filters to build)."""
import numpy as np

F32 = np.float32


def avg1d(a, h):
    """Running box average of half width h along axis 0 (avgVolume1D)."""
    a = np.asarray(a, F32)
    n1 = a.shape[0]
    sc = F32(1.0) / (F32(2.0) * F32(h) + F32(1.0))
    m = F32(h + 1.0) * a[0]
    for j in range(1, h + 1):
        m = m + a[min(j, n1 - 1)]
    b = np.empty_like(a)
    b[0] = m * sc
    for k in range(1, n1):
        k1, k2 = max(0, k - h - 1), min(n1 - 1, k + h)
        m = m + (a[k2] - a[k1])
        b[k] = m * sc
    return b


def smooth(illum, hxy, hz):
    """avgVolume3D (y, x, z) for ny > 1, avgVolume2D (x, z) otherwise."""
    v = np.asarray(illum, F32)
    if v.shape[0] > 1:
        v = avg1d(v, hxy)
    v = np.moveaxis(avg1d(np.moveaxis(v, 1, 0), hxy), 0, 1)
    v = np.moveaxis(avg1d(np.moveaxis(v, 2, 0), hz), 0, 2)
    return np.ascontiguousarray(v)


def compensate(illum, image, hxy=10, hz=10, amp_damping=1.0, damp_weight=0.07):
    """(damping factor, compensated image) as computeDamping + applyDamping."""
    v = smooth(illum, hxy, hz) if (hxy > 0 or hz > 0) else np.asarray(illum, F32)
    ny, nx, nz = v.shape
    average = (float(np.sum(v, dtype=np.float64)) / v.size) ** float(amp_damping)
    aa = (v.astype(np.float64) * (1.0 / average)).astype(F32)
    bb = np.exp(-aa)
    f = (1.0 / (average * (aa + F32(damp_weight) * bb).astype(np.float64))).astype(F32)
    nt = 10
    w = (F32(0.5) * (F32(1.0) - np.cos(F32(np.pi) * np.arange(nt, dtype=F32) / F32(nt)))).astype(F32)
    if ny > 1:
        for k in range(min(nt, ny)):
            f[k] *= w[k]
            f[ny - 1 - k] *= w[k] if ny - 1 - k > ny - nt - 1 else F32(1.0)
    for k in range(min(nt, nx)):
        f[:, k] *= w[k]
        if nx - 1 - k > nx - nt - 1:
            f[:, nx - 1 - k] *= w[k]
    return f, (np.asarray(image, F32) * f).astype(F32)
