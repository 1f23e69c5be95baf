"""The segment-parallel compact-FD pipeline (engine CFD on 3-D grids,
kernel_variant 8, or 6 with plain tile loads) against the FP64 oracle and the
split pipeline.

Its line solves run each segment of a line from zero entering states and
correct with the carried states, so its FP32 rounding differs from the
sequential band solve of FdEngine_cfd (bgprtm/FdEngine_cfd.cpp:24-297); the
bound is the one every compact-FD result here meets: within twice the
reference order's own FP32-vs-FP64 spread of the FP64 oracle.
"""
import numpy as np
import pytest
from scipy.ndimage import gaussian_filter

from konglong_b200 import workloads as W
from konglong_b200.propagator import Propagator, spread_coeffs
from konglong_b200.spec import ENGINE_CFD, FIELD_W1, ISO, TTI, VTI, PropSpec
from oracle import pyoracle as O
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu

SEG = 8  # kernel_variant: the segment-parallel pipeline (TMA tile loads where possible)


def _inputs(model, shape, seed, pml=9):
    nx, ny, nz = shape
    spec = PropSpec(nx=nx, ny=ny, nz=nz, dx=10.0, dy=10.0, dz=10.0, dt=0.001, engine=ENGINE_CFD, model_type=model,
                    nbnd=(pml,) * 6, vmax=4500.0)
    rng = np.random.default_rng(seed)
    sh = spec.shape
    m = dict(vel=(1800.0 + 2200.0 * rng.random(sh)).astype(np.float32))
    if model >= VTI:
        m["eps"] = (0.25 * rng.random(sh)).astype(np.float32)
        m["dl"] = (0.1 * rng.random(sh)).astype(np.float32)
    if model == TTI:
        th, ph = np.pi / 4 * rng.random(sh), 2 * np.pi * rng.random(sh)
        m["pjx"] = (-np.sin(th) * np.cos(ph)).astype(np.float32)
        m["pjy"] = (-np.sin(th) * np.sin(ph)).astype(np.float32)
    w0 = gaussian_filter(rng.standard_normal(sh), 1.5).astype(np.float32)
    w1 = gaussian_filter(rng.standard_normal(sh), 1.5).astype(np.float32)
    return spec, m, w0, w1


def _steps(x, spec, model, w0, w1, n):
    x.set_model(**model)
    x.put(0, w0)
    x.put(1, w1)
    for _ in range(n):
        x.kernel()
        x.update2nd()
        x.swap()
    return x.get(FIELD_W1 if isinstance(x, Propagator) else 1)


# several segments per axis with a last segment longer than the others, ragged
# 32-wide z tiles; TMA tile loads for (70, 45, 52) (nz % 4 == 0), plain loads
# for (33, 130, 17)
@pytest.mark.parametrize("model", [ISO, VTI, TTI])
@pytest.mark.parametrize("shape", [(70, 45, 52), (33, 130, 17)])
def test_operator_steps_within_the_conditioning_bound(model, shape):
    spec, m, w0, w1 = _inputs(model, shape, seed=30 + model, pml=6 if shape[2] < 24 else 9)
    spec.kernel_variant = SEG
    got = _steps(Propagator(spec), spec, m, w0, w1, 3)
    ref32 = _steps(O.Oracle(spec), spec, m, w0, w1, 3)
    exact = _steps(O.Oracle(spec, double=True), spec, m, w0, w1, 3)
    spread = rel_l2(ref32, exact)
    assert np.abs(exact).max() > 0
    assert rel_l2(got, exact) < 2 * spread + 1e-6, (rel_l2(got, exact), spread)


def test_tma_and_plain_tile_loads_bit_equal():
    """Variant 8 (TMA tile loads) and 6 (plain loads) run the same arithmetic."""
    shot = W.vti_cfd(scale=0.2, nt=40)
    out = []
    for variant in (SEG, 6):
        s = shot.spec
        s.kernel_variant = variant
        p = Propagator(s)
        p.set_model(**shot.model_arrays())
        k1, k2 = W.spread_band(s)
        src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
        p.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
        p.reset()
        p.modelling(40, -1, 1)
        out.append(p.get(FIELD_W1))
    np.testing.assert_array_equal(out[0], out[1])


@pytest.mark.parametrize("case", ["tti_q", "iso"])
def test_modelling_traces_vs_fp64(case):
    """Receiver traces of compact-FD shots: TTI + Q (the Q update in the fused x
    kernel) and ISO through the first-derivative path.  The TTI model is
    untilted: the reference's compact-FD TTI step grows without bound in tilted
    media (the compiled KernelCPU + FdEngine_cfd, and the oracle with it, pass
    1e5 within 20 steps in a homogeneous 30-degree tilt), so a long tilted run
    has no finite answer to compare with."""
    if case == "tti_q":
        shot = W.tti_q(scale=0.08, nt=150, engine=ENGINE_CFD)
        shot.pjx = np.zeros_like(shot.pjx)
        shot.pjy = np.zeros_like(shot.pjy)
    else:
        shot = W.vti_cfd(scale=0.1, nt=150)
        shot.spec.model_type = ISO
        shot.eps = shot.dl = None
    nts = 150
    s = shot.spec
    s.kernel_variant = SEG
    if s.use_q:
        cq0, cq, wq = W.q_coefficients(s.dt, shot.fpeak)
    res = []
    for x in (Propagator(s), O.Oracle(s), O.Oracle(s, double=True)):
        if s.use_q:
            x.set_q_coeffs(cq0, cq, wq)
        x.set_model(**shot.model_arrays())
        k1, k2 = W.spread_band(s)
        src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
        rcv = W.make_traceset(shot.rcv_pos, s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
        x.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
        x.set_extraction(rcv, nts)
        x.reset()
        x.modelling(nts, -1, 1)
        res.append(x.traces())
    got, want, exact = res
    assert np.abs(exact).max() > 0
    spread = rel_l2(want, exact)
    assert rel_l2(got, exact) < 2 * spread + 1e-5, (rel_l2(got, exact), spread)


def test_split_pipeline_agrees():
    """Variant 5 (split pipeline: sequential line solves and pointwise
    epilogues) and the segment-parallel pipeline give the same shot to within
    their FP32 rounding differences."""
    shot = W.vti_cfd(scale=0.15, nt=80)
    out = []
    for variant in (SEG, 5):
        s = shot.spec
        s.kernel_variant = variant
        p = Propagator(s)
        p.set_model(**shot.model_arrays())
        k1, k2 = W.spread_band(s)
        src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
        p.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
        p.reset()
        p.modelling(80, -1, 1)
        out.append(p.get(FIELD_W1))
    assert np.abs(out[1]).max() > 0
    assert rel_l2(out[0], out[1]) < 1e-3



def test_default_pipeline_2d_grid_and_derivative_path():
    """The default compact-FD pipeline on a 2-D grid (no y lines, no y faces)
    and on the Derivative path (CFD_BATCH), against the FP64 oracle."""
    for shape, engine in [((90, 1, 75), 1), ((70, 45, 52), 4)]:
        spec, m, w0, w1 = _inputs(VTI, shape, seed=11, pml=6)
        spec.engine = engine
        if shape[1] == 1:
            spec.nbnd = (6, 6, 0, 0, 6, 6)
        got = _steps(Propagator(spec), spec, m, w0, w1, 2)
        ref32 = _steps(O.Oracle(spec), spec, m, w0, w1, 2)
        exact = _steps(O.Oracle(spec, double=True), spec, m, w0, w1, 2)
        spread = rel_l2(ref32, exact)
        assert np.abs(exact).max() > 0
        assert rel_l2(got, exact) < 2 * spread + 1e-6, (shape, engine, rel_l2(got, exact), spread)
