"""The double-grid imaging oracle on the CPU: its copy map against the
reference's rules, the two line filters against known answers, and its
interleave / illumination interpolation against element-by-element
transcriptions of ImagingCorrelator::interleave2d / interleave3d
(bgprtm/ImagingCorrelator.cpp:447-507) and ImagingCondition::interpIllum
(bgprtm/ImagingCondition.cpp:759-808)."""
import numpy as np
import pytest

from oracle import ic_double_oracle as D


@pytest.mark.parametrize("dbl,want", [
    ((2, 1, 1), (dict(z=1, x=0, y=0, zx=0, zy=0, xy=0, zxy=0), 2)),
    ((2, 2, 1), (dict(z=1, x=2, y=0, zx=3, zy=0, xy=0, zxy=0), 4)),
    ((2, 2, 2), (dict(z=1, x=2, y=3, zx=4, zy=5, xy=6, zxy=7), 8)),
    ((1, 1, 1), (dict(z=0, x=0, y=0, zx=0, zy=0, xy=0, zxy=0), 1)),
])
def test_copy_map(dbl, want):
    assert D.copy_map(*dbl) == want


@pytest.mark.parametrize("n", [32, 33])
def test_half_shift_of_a_band_limited_line_is_its_midpoint_samples(n):
    rng = np.random.default_rng(n)
    x = np.arange(n, dtype=np.float64)
    a = rng.standard_normal(n // 2 - 1)
    ph = rng.uniform(0, 2 * np.pi, n // 2 - 1)
    f = lambda t: sum(a[k - 1] * np.cos(2 * np.pi * k * t / n + ph[k - 1]) for k in range(1, n // 2)) + 0.3
    line = np.broadcast_to(f(x), (3, 2, n)).copy()
    got = D.half_shift(line, 2)
    np.testing.assert_allclose(got, np.broadcast_to(f(x + 0.5), (3, 2, n)), atol=1e-12)
    # along x and y too
    np.testing.assert_allclose(D.half_shift(np.moveaxis(line, 2, 1), 1), np.moveaxis(np.broadcast_to(
        f(x + 0.5), (3, 2, n)), 2, 1), atol=1e-12)


def test_high_cut_passes_the_band_below_high_and_removes_nyquist():
    n = 40
    x = np.arange(n)
    low = np.cos(2 * np.pi * 5 * x / n) + 0.5 * np.sin(2 * np.pi * 11 * x / n)  # 11 / 20 = 0.55 of Nyquist
    np.testing.assert_allclose(D.high_cut(low[None, None, :], 2, 0.7)[0, 0], low, atol=1e-12)
    nyq = np.cos(np.pi * x)
    np.testing.assert_allclose(D.high_cut(nyq[None, None, :], 2, 0.7)[0, 0], 0.0, atol=1e-12)
    mid = np.cos(2 * np.pi * 17 * x / n)  # 0.85 of Nyquist: weight 0.5 (1 + cos(pi 0.15 / 0.3)) = 0.5
    np.testing.assert_allclose(D.high_cut(mid[None, None, :], 2, 0.7)[0, 0], 0.5 * mid, atol=1e-12)


def _interleave_loops(cubes, dz, dx, dy):
    """interleave3d / interleave2d transcribed element by element."""
    iv, nloop = D.copy_map(dz, dx, dy)
    ny, nx, nz = cubes[0].shape
    nz2, nx2 = nz * dz, nx * dx
    out = np.zeros(ny * dy * nx2 * nz2, np.float32)
    b = [np.asarray(c).ravel() for c in cubes]
    for iy in range(ny):
        for ix in range(nx):
            for iz in range(nz):
                idd = (iy * nx + ix) * nz + iz
                if nloop == 8:
                    iy1, iy2, ix1, ix2, iz1, iz2 = 2 * iy, 2 * iy + 1, 2 * ix, 2 * ix + 1, 2 * iz, 2 * iz + 1
                    out[(iy1 * nx2 + ix1) * nz2 + iz1] = b[0][idd]
                    out[(iy1 * nx2 + ix1) * nz2 + iz2] = b[iv["z"]][idd]
                    out[(iy1 * nx2 + ix2) * nz2 + iz1] = b[iv["x"]][idd]
                    out[(iy2 * nx2 + ix1) * nz2 + iz1] = b[iv["y"]][idd]
                    out[(iy1 * nx2 + ix2) * nz2 + iz2] = b[iv["zx"]][idd]
                    out[(iy2 * nx2 + ix1) * nz2 + iz2] = b[iv["zy"]][idd]
                    out[(iy2 * nx2 + ix2) * nz2 + iz1] = b[iv["xy"]][idd]
                    out[(iy2 * nx2 + ix2) * nz2 + iz2] = b[iv["zxy"]][idd]
                else:  # interleave2d on one xz plane (ny == 1)
                    ndx = 2 if iv["x"] else 1
                    ix1, ix2 = ix * ndx, ix * ndx + ndx - 1
                    out[ix1 * nz2 + iz * 2] = b[0][idd]
                    out[ix1 * nz2 + iz * 2 + 1] = b[iv["z"]][idd]
                    if iv["zx"]:
                        out[ix2 * nz2 + iz * 2] = b[iv["x"]][idd]
                        out[ix2 * nz2 + iz * 2 + 1] = b[iv["zx"]][idd]
    return out.reshape(ny * dy, nx2, nz2)


@pytest.mark.parametrize("shape,dbl", [((3, 4, 5), (2, 2, 2)), ((1, 6, 7), (2, 2, 1)), ((1, 5, 4), (2, 1, 1))])
def test_interleave_matches_the_reference_loops(shape, dbl):
    _, nloop = D.copy_map(*dbl)
    rng = np.random.default_rng(3)
    cubes = [rng.standard_normal(shape).astype(np.float32) for _ in range(nloop)]
    np.testing.assert_array_equal(D.interleave(cubes, *dbl), _interleave_loops(cubes, *dbl))


def _interp_illum_loops(a, dz, dx, dy):
    """interpIllum transcribed element by element (float32, its term order)."""
    ny, nx, nz = a.shape
    nx2, nz2 = nx * dx, nz * dz
    out = np.zeros(ny * dy * nx2 * nz2, np.float32)
    v = a.ravel()
    f = np.float32
    for iy in range(ny):
        for ix in range(nx):
            iy1, iy2 = iy * dy, iy * dy + (0 if dy == 1 else 1)
            ix1, ix2 = ix * dx, ix * dx + (0 if dx == 1 else 1)
            for iz in range(nz):
                iz1, iz2 = iz * dz, iz * dz + (0 if dz == 1 else 1)
                idd = (iy * nx + ix) * nz + iz
                ids = [(iy1 * nx2 + ix1) * nz2 + iz1, (iy2 * nx2 + ix1) * nz2 + iz1, (iy1 * nx2 + ix2) * nz2 + iz1,
                       (iy1 * nx2 + ix1) * nz2 + iz2, (iy2 * nx2 + ix1) * nz2 + iz2, (iy1 * nx2 + ix2) * nz2 + iz2,
                       (iy2 * nx2 + ix2) * nz2 + iz1, (iy2 * nx2 + ix2) * nz2 + iz2]
                yp, xp, zp = min(iy + 1, ny - 1), min(ix + 1, nx - 1), min(iz + 1, nz - 1)
                g = lambda y, x, z: v[(y * nx + x) * nz + z]
                c = v[idd]
                out[ids[0]] = c
                out[ids[1]] = f(0.5) * (g(iy, ix, iz) + g(yp, ix, iz))
                out[ids[2]] = f(0.5) * (g(iy, ix, iz) + g(iy, xp, iz))
                out[ids[3]] = f(0.5) * (g(iy, ix, iz) + g(iy, ix, zp))
                out[ids[4]] = f(0.25) * (g(iy, ix, iz) + g(iy, ix, zp) + g(yp, ix, iz) + g(yp, ix, zp))
                out[ids[5]] = f(0.25) * (g(iy, ix, iz) + g(iy, ix, zp) + g(iy, xp, iz) + g(iy, xp, zp))
                out[ids[6]] = f(0.25) * (g(iy, ix, iz) + g(yp, ix, iz) + g(iy, xp, iz) + g(yp, xp, iz))
                out[ids[7]] = f(0.125) * (g(iy, ix, iz) + g(yp, ix, iz) + g(iy, xp, iz) + g(iy, ix, zp) +
                                          g(yp, ix, zp) + g(yp, xp, iz) + g(iy, xp, zp) + g(yp, xp, zp))
    return out.reshape(ny * dy, nx2, nz2)


@pytest.mark.parametrize("shape,dbl", [((3, 4, 5), (2, 2, 2)), ((1, 6, 7), (2, 2, 1)), ((1, 5, 4), (2, 1, 1))])
def test_interp_illum_matches_the_reference_loops(shape, dbl):
    a = np.random.default_rng(4).random(shape).astype(np.float32)
    np.testing.assert_array_equal(D.interp_illum(a, *dbl), _interp_illum_loops(a, *dbl))
