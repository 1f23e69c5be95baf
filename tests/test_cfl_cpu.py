"""Known answers for the time-step rule (ModelPrepare::calcDeltaTime,
bgprtm/ModelPrepare.cpp:647-891) and the FD8 k1max (FdEngine_fd::get_k1max,
bgprtm/FdEngine_fd.cpp:69-81), worked out by hand on homogeneous models.

Each expected value below is written as the arithmetic a reader can redo on
paper; `cfl_dt` must reproduce it for the FD8 (k1max from the Taylor table)
and compact-FD (k1max = pi) engines, for ISO / VTI / TTI, with density and
with the Q rescale.
"""
import math

import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200.spec import ENGINE_CFD, ENGINE_FD8, ISO, TTI, VTI, PropSpec


def spec(engine, model, n=12, d=10.0, use_q=0):
    s = PropSpec(nx=n, ny=n, nz=n, dx=d, dy=d, dz=d, dt=1e-3, engine=engine, model_type=model,
                 nbnd=(0,) * 6, vmax=3000.0)
    s.use_q = use_q
    return s


def const(v, n=12):
    return np.full((n, n, n), v, np.float32)


# 8th-order Taylor second-derivative weights c0 = -205/72, c1..c4 = 8/5, -1/5,
# 8/315, -1/560: sum2 = -c0 + 2 c1 - 2 c2 + 2 c3 - 2 c4 (alternating signs),
# k1max = sqrt(sum2) * 1.01
SUM2 = 205 / 72 + 2 * 8 / 5 + 2 * 1 / 5 + 2 * 8 / 315 + 2 * 1 / 560   # = 6.5015873...
K1_FD8 = math.sqrt(SUM2) * 1.01                                       # = 2.5753193...
K1_PI = math.pi


def test_fd8_k1max_is_the_taylor_table_bound():
    assert SUM2 == pytest.approx(6.50158730, rel=1e-8)
    assert W.fd8_k1max() == pytest.approx(K1_FD8, rel=1e-6)


@pytest.mark.parametrize("engine,k1", [(ENGINE_FD8, K1_FD8), (ENGINE_CFD, K1_PI)])
def test_iso_homogeneous(engine, k1):
    # lambda = v sqrt(3 / d^2) = 2500 sqrt(0.03) = 433.0127 1/s ; dt = 2 / k1 / lambda
    lam = 2500.0 * math.sqrt(3 / 100.0)
    want = 2.0 / k1 / lam
    assert W.cfl_dt(spec(engine, ISO), const(2500.0)) == pytest.approx(want, rel=1e-6)


@pytest.mark.parametrize("engine,k1", [(ENGINE_FD8, K1_FD8), (ENGINE_CFD, K1_PI)])
def test_vti_homogeneous(engine, k1):
    # e = 0.2, d = 0.1, v = 3000, 1/d^2 = 0.01:  h2 = 0.02, z2 = 0.01
    # tmp = 1.4 * 0.02 + 0.01 = 0.038 ; disc = 0.038^2 - 8 * 0.1 * 0.02 * 0.01 = 0.001284
    # lambda = 3000 sqrt((0.038 + sqrt(0.001284)) / 2) ; dt = 2 / k1 / lambda / sqrt(1.4)
    lam = 3000.0 * math.sqrt((0.038 + math.sqrt(0.001284)) / 2)
    want = 2.0 / k1 / lam / math.sqrt(1.4)
    got = W.cfl_dt(spec(engine, VTI), const(3000.0), const(0.2), const(0.1))
    assert got == pytest.approx(want, rel=1e-6)


def test_tti_untilted_axis_takes_the_largest_axis_combination():
    # theta = 0: the rotated wavenumbers are the grid's (rx = ry = rz = 0.01).
    # ic runs over the 7 non-empty subsets of (z, x, y); for e = 0.2, d = 0.1:
    #   z only      : t1 = 0.01,            lambda = v * 0.1
    #   x or y only : t1 = 1.4 * 0.01,      lambda = v * sqrt(0.014)
    #   x + y       : t1 = 1.4 * 0.02,      lambda = v * sqrt(0.028)
    #   z + x, z + y: t1 = 0.024, disc = 0.024^2 - 8*0.1*0.01*0.01 = 0.000496
    #   all three   : t1 = 0.038, disc = 0.001284 (the VTI value)
    v = 3000.0
    cands = [0.1, math.sqrt(0.014), math.sqrt(0.028),
             math.sqrt((0.024 + math.sqrt(0.000496)) / 2), math.sqrt((0.038 + math.sqrt(0.001284)) / 2)]
    lam = v * max(cands)
    want = 2.0 / K1_FD8 / lam / math.sqrt(1.4)
    got = W.cfl_dt(spec(ENGINE_FD8, TTI), const(v), const(0.2), const(0.1), const(0.0), const(0.0))
    assert got == pytest.approx(want, rel=1e-6)


def test_tti_axis_along_x_on_a_stretched_grid():
    # theta = 90 deg, phi = 0 (pjx = -1, pjy = 0): cos phi = 1, sin phi = 0,
    # cos theta = 0, sin theta = 1.  With dx = 10, dy = 20, dz = 40:
    #   rx = (-1/dz)^2 = 1/1600, ry = (1/dy)^2 = 1/400, rz = (1/dx)^2 = 1/100
    # e = d = 0 (isotropic values through the TTI rule): every combination
    # gives lambda = v sqrt(sum of its terms); the largest is all three.
    s = PropSpec(nx=12, ny=12, nz=12, dx=10.0, dy=20.0, dz=40.0, dt=1e-3, engine=ENGINE_FD8, model_type=TTI,
                 nbnd=(0,) * 6, vmax=3000.0)
    v = 2000.0
    lam = v * math.sqrt(1 / 1600 + 1 / 400 + 1 / 100)
    want = 2.0 / K1_FD8 / lam
    got = W.cfl_dt(s, const(v), const(0.0), const(0.0), const(-1.0), const(0.0))
    assert got == pytest.approx(want, rel=1e-5)


def test_density_scales_lambda_and_the_minimum():
    # ISO, v = 2000, rho = 2.25 everywhere except one cell of 1.0:
    # lambda_max = 2000 * sqrt(2.25) * sqrt(0.03) (the dense cells),
    # dt = 2 / k1 / lambda_max * sqrt(min rho) = 2 / k1 / (2000 * 1.5 * sqrt(0.03)) * 1
    rho = const(2.25)
    rho[3, 4, 5] = 1.0
    want = 2.0 / K1_FD8 / (2000.0 * 1.5 * math.sqrt(0.03)) * 1.0
    got = W.cfl_dt(spec(ENGINE_FD8, ISO), const(2000.0), rho=rho)
    assert got == pytest.approx(want, rel=1e-6)


def test_q_rescale():
    # max(1/Q) = 1/30, maxfreq = 60 Hz, qref = maxfreq / 3 = 20 Hz:
    # rescale = 1 - (1/30) (3 + (2/pi) ln 3) = 1 - 0.1 - 0.0233133... = 0.8766867
    invq = const(1 / 100.0)
    invq[0, 0, 0] = 1 / 30.0
    base = W.cfl_dt(spec(ENGINE_FD8, ISO), const(2500.0))
    got = W.cfl_dt(spec(ENGINE_FD8, ISO, use_q=1), const(2500.0), invq=invq, maxfreq=60.0)
    rescale = 1 - (1 / 30.0) * (3 + 2 / math.pi * math.log(3.0))
    assert rescale == pytest.approx(0.8766867, rel=1e-6)
    assert got == pytest.approx(base * rescale, rel=1e-6)
