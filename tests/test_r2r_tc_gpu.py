"""FFTWR2R line operators on the tensor cores (split-TF32 tcgen05 kernel,
kernel_variant 0: z lines as a K-major product, x and y lines with the volume
as an MN-major operand) against the same operators as FP32 cuBLAS GEMMs
(kernel_variant 1) and against the FP64 oracle (FdEngine_r2r's line matrices,
bgprtm/FdEngine_r2r.cpp).  Line lengths 20 to 512 cover one and two
256-column accumulator halves and a last 16-column pad; 20 x 24 = 480 z lines
and 20 x 28 = 560 y columns leave partial last 128-line tiles; a grid whose nz
is not a multiple of 4 takes the cuBLAS products on every axis."""
import numpy as np
import pytest

from konglong_b200.propagator import Propagator
from konglong_b200.spec import ENGINE_FFTV, ENGINE_R2C, ENGINE_R2R, FIELD_W1, ISO, TTI, VTI
from oracle import pyoracle as O
from tests.conftest import rel_l2
from tests.golden_inputs import case_inputs

pytestmark = pytest.mark.gpu


def _steps(x, m, w0, w1, n):
    x.set_model(**m)
    x.put(0, w0)
    x.put(1, w1)
    for _ in range(n):
        x.kernel()
        x.update2nd()
        x.swap()
    return x.get(FIELD_W1 if isinstance(x, Propagator) else 1)


@pytest.mark.parametrize("nz", [28, 200, 400, 512])
@pytest.mark.parametrize("model", [ISO, VTI, TTI])
def test_tensor_core_z_lines_match_fp32_gemm_and_fp64(nz, model):
    c = dict(engine=ENGINE_R2R, model=model, shape=(20, 24, nz), pml=6, seed=70 + model)
    spec, m, w0, w1 = case_inputs(c)
    out = {}
    for variant in (0, 1):
        spec.kernel_variant = variant
        out[variant] = _steps(Propagator(spec), m, w0, w1, 2)
    assert np.abs(out[1]).max() > 0
    assert rel_l2(out[0], out[1]) < 2e-6, rel_l2(out[0], out[1])
    if nz <= 200:  # the FP64 oracle at the sizes it finishes in seconds
        exact = _steps(O.Oracle(spec, double=True), m, w0, w1, 2)
        ref32 = _steps(O.Oracle(spec), m, w0, w1, 2)
        assert rel_l2(out[0], exact) < 2 * rel_l2(ref32, exact) + 1e-6


@pytest.mark.parametrize("shape", [(300, 20, 36), (36, 300, 20), (40, 30, 30)])
def test_tensor_core_x_y_lines(shape):
    c = dict(engine=ENGINE_R2R, model=VTI, shape=shape, pml=6, seed=77)
    spec, m, w0, w1 = case_inputs(c)
    out = {}
    for variant in (0, 1):
        spec.kernel_variant = variant
        out[variant] = _steps(Propagator(spec), m, w0, w1, 2)
    assert np.abs(out[1]).max() > 0
    assert rel_l2(out[0], out[1]) < 2e-6, rel_l2(out[0], out[1])


@pytest.mark.parametrize("engine", [ENGINE_R2C, ENGINE_FFTV])
@pytest.mark.parametrize("shape", [(20, 24, 28), (21, 25, 36), (36, 20, 300)])
def test_tensor_core_spectral_circulants(engine, shape):
    """FFTWR2C / FFTV: each axis derivative as its circulant line matrix on the
    tensor cores (kernel_variant 0) against cuFFT transforms with the bin
    product (kernel_variant 1); odd lines carry the pass's isign on their last
    bin (FdEngine_r2c::fftderiv1_r2c)."""
    c = dict(engine=engine, model=VTI, shape=shape, pml=6, seed=78)
    spec, m, w0, w1 = case_inputs(c)
    out = {}
    for variant in (0, 1):
        spec.kernel_variant = variant
        out[variant] = _steps(Propagator(spec), m, w0, w1, 2)
    assert np.abs(out[1]).max() > 0
    assert rel_l2(out[0], out[1]) < 3e-6, rel_l2(out[0], out[1])
