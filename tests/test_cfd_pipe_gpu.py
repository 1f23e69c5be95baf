"""The pipelined persistent x / y line solves (kernel_variant 10: one CTA per
SM, a ring of TMA tile buffers, the right-hand side formed inside the
forward elimination) against the default split pipeline, whose x / y solves
form the right-hand sides in a separate pass (bgprtm/FdEngine_cfd.cpp
banmul + banbks).  Both compute every row with the same roundings, so the
fields must agree bit for bit: 3 to 8 buffers in the ring (lines of 512,
300, 130 and 45 points), ragged 32-line z tiles, ISO / VTI / TTI, the
Derivative path, density, and a TTI + Q modelling run.
"""
import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200.propagator import Propagator, spread_coeffs
from konglong_b200.spec import ENGINE_CFD, ENGINE_CFDB, FIELD_W0, FIELD_W1, ISO, TTI, VTI
from tests.golden_inputs import case_inputs

pytestmark = pytest.mark.gpu

PIPE = 10


def _kernel_steps(spec, m, w0, w1, variant, n=3):
    spec.kernel_variant = variant
    p = Propagator(spec)
    p.set_model(**m)
    p.put(0, w0)
    p.put(1, w1)
    for _ in range(n):
        p.kernel()
        p.update2nd()
        p.swap()
    return p.get(FIELD_W0), p.get(FIELD_W1)


@pytest.mark.parametrize("model", [ISO, VTI, TTI])
@pytest.mark.parametrize("shape", [(512, 20, 36), (40, 300, 44), (130, 45, 52), (33, 18, 68)])
def test_pipelined_line_solves_bit_equal(model, shape):
    c = dict(engine=ENGINE_CFD, model=model, shape=shape, pml=6, seed=50 + model)
    spec, m, w0, w1 = case_inputs(c)
    got = _kernel_steps(spec, m, w0, w1, PIPE)
    want = _kernel_steps(spec, m, w0, w1, 0)
    assert np.abs(want[1]).max() > 0
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("engine,rho", [(ENGINE_CFDB, False), (ENGINE_CFD, True), (ENGINE_CFDB, True)])
def test_pipelined_line_solves_derivative_path_and_density(engine, rho):
    c = dict(engine=engine, model=TTI, shape=(64, 40, 48), pml=6, seed=61, rho=rho)
    spec, m, w0, w1 = case_inputs(c)
    got = _kernel_steps(spec, m, w0, w1, PIPE)
    want = _kernel_steps(spec, m, w0, w1, 0)
    for a, b in zip(got, want):
        np.testing.assert_array_equal(a, b)


def test_pipelined_line_solves_tti_q_modelling():
    shot = W.tti_q(scale=0.06, nt=60, engine=ENGINE_CFD)
    shot.pjx = np.zeros_like(shot.pjx)
    shot.pjy = np.zeros_like(shot.pjy)
    s = shot.spec
    cq0, cq, wq = W.q_coefficients(s.dt, shot.fpeak)
    out = []
    for variant in (PIPE, 0):
        s.kernel_variant = variant
        p = Propagator(s)
        p.set_q_coeffs(cq0, cq, wq)
        p.set_model(**shot.model_arrays())
        k1, k2 = W.spread_band(s)
        src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
        rcv = W.make_traceset(shot.rcv_pos, s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
        p.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
        p.set_extraction(rcv, 60)
        p.reset()
        p.modelling(60, -1, 1)
        out.append((p.get(FIELD_W1), p.traces()))
    assert np.abs(out[1][1]).max() > 0
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
