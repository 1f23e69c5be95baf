"""CPU oracle of the double-grid IMAGE1 imaging condition (test infrastructure
only: the tests import it as the checker, nothing else runs it).

Float64 numpy restatement of what one imaging step computes on the doubled
grid (ImagingCondition::stackImageInterp, bgprtm/ImagingCondition.cpp:104-141):

* applyFFTV (:169-178): a high cut along each doubled axis, in place, on the
  tapered source and receiver fields; interp (:1084-1111) /
  ImagingCorrelator::interp (bgprtm/ImagingCorrelator.cpp:509-517): the copies
  half-shifted along z, x, y from copy 0, then zx, zy, xy, zxy from the z / x /
  zx copies.  Both filters are libfftv's (HIGHTAPE, SHIFTHALF), which is not in
  the reference tree: they are restated from their use.  SHIFTHALF must give the
  field at x + d/2, because interleave puts its copy on the odd points of the
  doubled grid (i.e. between x_i and x_{i+1}); the restatement is the
  band-limited shift (bin j times e^{i pi j / n}, the Nyquist bin of an even
  line dropped because its cosine vanishes at the midpoints).  HIGHTAPE's shape
  is not published; the restatement passes wavenumbers up to `high` of Nyquist
  and rolls off to zero at Nyquist with a cosine.  Parity of these two filters
  is therefore unpinned (known answers only: a band-limited line shifted by
  half a step equals its samples at the midpoints, a band below `high` passes
  unchanged).
* ImagingCorrelator::imaging1 (:363-372): image cube i += copy i of the source
  x copy i of the receiver (crossone, isign +1).
* interleave2d / interleave3d (:440-507) and ImagingCondition::interpIllum
  (bgprtm/ImagingCondition.cpp:759-808), restated literally (index formulas and
  write order).
"""
import numpy as np


def copy_map(dz, dx, dy):
    """ImagingCorrelator's copy numbers (ivz, ivx, ivy, ivzx, ivzy, ivxy, ivzxy) and
    nloop (bgprtm/ImagingCorrelator.cpp:57-74)."""
    ivz, ivx, ivy, ivzx, ivzy, ivxy, ivzxy = 1, 2, 3, 4, 5, 6, 7
    if dy == 1:
        if dz == 1:
            ivx = 1
        else:
            ivz, ivx, ivzx = 1, 2, 3
    elif dx == 1:
        if dz == 1:
            ivy = 1
        else:
            ivz, ivy, ivzy = 1, 2, 3
    elif dz == 1:
        ivx, ivy, ivxy = 1, 2, 3
    if dy == 1:
        ivy = ivxy = ivzy = ivzxy = 0
    if dx == 1:
        ivx = ivxy = ivzx = ivzxy = 0
    if dz == 1:
        ivz = ivzx = ivzy = ivzxy = 0
    nloop = 8 if ivzxy else 4 if ivzx else 2 if ivz else 1
    return dict(z=ivz, x=ivx, y=ivy, zx=ivzx, zy=ivzy, xy=ivxy, zxy=ivzxy), nloop


# volumes are [ny][nx][nz]: numpy axis of z, x, y
AXIS = {"z": 2, "x": 1, "y": 0}


def half_shift(a, axis):
    """Band-limited value at x + d/2 of every line along `axis`."""
    a = np.asarray(a, np.float64)
    n = a.shape[axis]
    F = np.fft.rfft(a, axis=axis)
    j = np.arange(F.shape[axis])
    ph = np.exp(1j * np.pi * j / n)
    if n % 2 == 0:
        ph[-1] = 0.0
    shape = [1] * a.ndim
    shape[axis] = -1
    return np.fft.irfft(F * ph.reshape(shape), n=n, axis=axis)


def high_cut(a, axis, high):
    """Wavenumbers above `high` of Nyquist rolled off to zero at Nyquist (cosine)."""
    a = np.asarray(a, np.float64)
    n = a.shape[axis]
    F = np.fft.rfft(a, axis=axis)
    q = np.arange(F.shape[axis]) / (0.5 * n)
    w = np.where(q <= high, 1.0, 0.5 * (1.0 + np.cos(np.pi * np.minimum((q - high) / (1.0 - high), 1.0))))
    shape = [1] * a.ndim
    shape[axis] = -1
    return np.fft.irfft(F * w.reshape(shape), n=n, axis=axis)


def copies(f, dz, dx, dy, high_z, high_xy):
    """The filtered field and its half-shifted copies, indexed by copy number."""
    f = np.asarray(f, np.float64)
    if dz > 1:
        f = high_cut(f, AXIS["z"], high_z)
    if dx > 1:
        f = high_cut(f, AXIS["x"], high_xy)
    if dy > 1:
        f = high_cut(f, AXIS["y"], high_xy)
    iv, nloop = copy_map(dz, dx, dy)
    c = {0: f}
    for name, src, ax in (("z", 0, "z"), ("x", 0, "x"), ("y", 0, "y"), ("zx", iv["z"], "x"),
                          ("zy", iv["z"], "y"), ("xy", iv["x"], "y"), ("zxy", iv["zx"], "y")):
        if iv[name]:
            c[iv[name]] = half_shift(c[src], AXIS[ax])
    return [c[i] for i in range(nloop)]


def image_step(S, R, dz, dx, dy, high_z=0.9, high_xy=0.7):
    """Image cubes (nloop of them) of one imaging step, and the filtered source
    field the illumination takes."""
    cs = copies(S, dz, dx, dy, high_z, high_xy)
    cr = copies(R, dz, dx, dy, high_z, high_xy)
    return [s * r for s, r in zip(cs, cr)], cs[0]


def interleave(cubes, dz, dx, dy):
    """The image cubes on the doubled grid [ny*dy][nx*dx][nz*dz]
    (interleave3d for 8 cubes, interleave2d otherwise: every xz plane)."""
    iv, nloop = copy_map(dz, dx, dy)
    ny, nx, nz = cubes[0].shape
    out = np.zeros((ny * dy, nx * dx, nz * dz), np.asarray(cubes[0]).dtype)
    if nloop == 1:
        return np.array(cubes[0])
    out[0::dy, 0::dx, 0::dz] = cubes[0]
    out[0::dy, 0::dx, 1::dz] = cubes[iv["z"]]
    if nloop == 8:
        out[0::dy, 1::dx, 0::dz] = cubes[iv["x"]]
        out[1::dy, 0::dx, 0::dz] = cubes[iv["y"]]
        out[0::dy, 1::dx, 1::dz] = cubes[iv["zx"]]
        out[1::dy, 0::dx, 1::dz] = cubes[iv["zy"]]
        out[1::dy, 1::dx, 0::dz] = cubes[iv["xy"]]
        out[1::dy, 1::dx, 1::dz] = cubes[iv["zxy"]]
    elif iv["zx"]:
        out[0::dy, 1::dx, 0::dz] = cubes[iv["x"]]
        out[0::dy, 1::dx, 1::dz] = cubes[iv["zx"]]
    return out


def interp_illum(a, dz, dx, dy):
    """ImagingCondition::interpIllum: the eight targets of every cell in the
    reference's order (on an axis that is not doubled the odd index equals the
    even one, so later targets overwrite earlier ones)."""
    a = np.asarray(a, np.float32)
    ny, nx, nz = a.shape
    if dz * dx * dy == 1:
        return a.copy()
    out = np.zeros((ny * dy, nx * dx, nz * dz), np.float32)
    iy, ix, iz = np.arange(ny), np.arange(nx), np.arange(nz)
    yp, xp, zp = np.minimum(iy + 1, ny - 1), np.minimum(ix + 1, nx - 1), np.minimum(iz + 1, nz - 1)
    y1, y2 = iy * dy, iy * dy + (dy - 1)
    x1, x2 = ix * dx, ix * dx + (dx - 1)
    z1, z2 = iz * dz, iz * dz + (dz - 1)

    def at(y, x, z):
        return a[np.ix_(y, x, z)]

    def put(y, x, z, v):
        out[np.ix_(y, x, z)] = v

    f = np.float32
    A = at(iy, ix, iz)
    put(y1, x1, z1, A)
    put(y2, x1, z1, f(0.5) * (A + at(yp, ix, iz)))
    put(y1, x2, z1, f(0.5) * (A + at(iy, xp, iz)))
    put(y1, x1, z2, f(0.5) * (A + at(iy, ix, zp)))
    put(y2, x1, z2, f(0.25) * (A + at(iy, ix, zp) + at(yp, ix, iz) + at(yp, ix, zp)))
    put(y1, x2, z2, f(0.25) * (A + at(iy, ix, zp) + at(iy, xp, iz) + at(iy, xp, zp)))
    put(y2, x2, z1, f(0.25) * (A + at(yp, ix, iz) + at(iy, xp, iz) + at(yp, xp, iz)))
    put(y2, x2, z2, f(0.125) * (A + at(yp, ix, iz) + at(iy, xp, iz) + at(iy, ix, zp) + at(yp, ix, zp) +
                                at(yp, xp, iz) + at(iy, xp, zp) + at(yp, xp, zp)))
    return out
