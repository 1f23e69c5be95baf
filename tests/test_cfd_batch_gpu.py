"""Engine CFD_BATCH (the Derivative path of Propagator::kernel: Derivative_cfd
line solves, Boundary's per-axis PML, the divergence plan of iswitch) on the
GPU against the oracle: operator steps for ISO / VTI / TTI and VTI modelling
traces.  Compact FD amplifies FP32 rounding (band LU pivots down to ~0.016), so
the bound is twice the oracle's own FP32-vs-FP64 spread, as for Engine CFD."""
import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200.propagator import Propagator, spread_coeffs
from konglong_b200.spec import ENGINE_CFDB, FIELD_W1
from oracle import pyoracle as O
from tests.conftest import rel_l2
from tests.golden_inputs import case_inputs
from tests.test_gpu_parity import _modelling

pytestmark = pytest.mark.gpu


def _steps(x, n):
    for _ in range(n):
        x.kernel()
        x.update2nd()
        x.swap()


@pytest.mark.parametrize("model", [1, 2, 3])
def test_cfd_batch_operator_steps(model):
    c = dict(engine=ENGINE_CFDB, model=model, shape=(24, 20, 28), pml=6, steps=3, seed=41)
    spec, m, w0, w1 = case_inputs(c)
    out = []
    for x in (Propagator(spec), O.Oracle(spec), O.Oracle(spec, double=True)):
        x.set_model(**m)
        x.put(0, w0)
        x.put(1, w1)
        _steps(x, 3)
        out.append(np.asarray(x.get(FIELD_W1 if isinstance(x, Propagator) else 1), np.float64).ravel())
    got, want, exact = out
    spread = rel_l2(want, exact)
    assert np.abs(exact).max() > 0 and spread < 5e-3
    assert rel_l2(got, exact) < 2 * spread + 1e-6


def test_cfd_batch_modelling_traces():
    nts = 200
    shot = W.vti_cfd(scale=0.1, nt=nts)
    shot.spec.engine = ENGINE_CFDB
    got = _modelling(shot, Propagator(shot.spec), spread_coeffs, nts)
    want = _modelling(shot, O.Oracle(shot.spec), spread_coeffs, nts)
    exact = _modelling(shot, O.Oracle(shot.spec, double=True), spread_coeffs, nts)
    assert np.abs(exact).max() > 0
    spread = rel_l2(want, exact)
    assert rel_l2(got, exact) < 2 * spread + 1e-5
