"""The compact-FD z line solve fused with the interior cells of the pointwise
epilogue that follows it (kernel_variant 9) against the default split
pipeline (the z solves and the epilogues as separate launches).

The fused kernels keep the raw z derivative of their 32 lines in shared
memory and run the epilogue's per-cell arithmetic on the interior cells
(PML cells get the raw value stored for the PML face-box launches), so every
field must come out with the same bits: the gradient pass of ISO / VTI / TTI with and
without density (bgprtm/KernelCPU.cpp ScalarVTI / ScalarTTI, PML round 1),
the divergence pass's accumulation with PML round 2 and the leapfrog update
(Propagator::update2nd), the Derivative path (CFD_BATCH) with its
divergence-pass plan, 2-D grids, and ragged 32-line tiles.  TTI + Q runs the
fused gradient pass and the separate divergence epilogue (its Q update stays
unfused).
"""
import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200.propagator import Propagator, spread_coeffs
from konglong_b200.spec import ENGINE_CFD, ENGINE_CFDB, FIELD_W0, FIELD_W1, ISO, TTI, VTI
from tests.golden_inputs import case_inputs

pytestmark = pytest.mark.gpu

FUSED = 9


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
@pytest.mark.parametrize("engine", [ENGINE_CFD, ENGINE_CFDB])
@pytest.mark.parametrize("rho", [False, True])
@pytest.mark.parametrize("shape", [(33, 18, 70), (37, 1, 44)])
def test_fused_z_epilogue_bit_equal(model, engine, rho, shape):
    c = dict(engine=engine, model=model, shape=shape, pml=6, seed=40 + model + 3 * rho, rho=rho)
    spec, m, w0, w1 = case_inputs(c)
    if shape[1] == 1:
        spec.nbnd = (6, 6, 0, 0, 6, 6)
    fused = _kernel_steps(spec, m, w0, w1, FUSED)
    split = _kernel_steps(spec, m, w0, w1, 0)
    assert np.abs(split[1]).max() > 0
    for a, b in zip(fused, split):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("case", ["vti", "tti_q"])
def test_fused_z_epilogue_modelling_bit_equal(case):
    """Whole modelling runs (leapfrog update in the divergence epilogue, or
    the Q update after a fused gradient pass) with injection and traces."""
    if case == "vti":
        shot = W.vti_cfd(scale=0.12, nt=60)
    else:
        shot = W.tti_q(scale=0.06, nt=60, engine=ENGINE_CFD)
        shot.pjx = np.zeros_like(shot.pjx)
        shot.pjy = np.zeros_like(shot.pjy)
    s = shot.spec
    if s.use_q:
        cq0, cq, wq = W.q_coefficients(s.dt, shot.fpeak)
    out = []
    for variant in (FUSED, 0):
        s.kernel_variant = variant
        p = Propagator(s)
        if s.use_q:
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
