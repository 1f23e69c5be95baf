"""CPU-side checks of the drop-in boundary: the C-ABI library loads, exports
every entry point include/rtm_b200.h declares, and its host-side set-up
(spread coefficients, argument validation) behaves like the reference's."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from konglong_b200 import _lib
from oracle import pyoracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "rtm_b200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char \*)\s*(rtm_[a-z0-9_]+)\s*\(", txt, re.M)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    syms = header_symbols()
    assert len(syms) >= 25
    for s in syms:
        assert hasattr(L, s), s
    assert sorted(_lib.EXPORTS) == syms


def test_spread_coeffs_match_oracle():
    from konglong_b200.propagator import spread_coeffs
    rng = np.random.default_rng(3)
    for _ in range(200):
        n = int(rng.integers(2, 300))
        x = float(rng.uniform(0, n - 1))
        k1 = float(rng.uniform(0.05, 0.5))
        k2 = float(rng.uniform(k1, 0.5)) if rng.random() < 0.5 else k1
        nl = int(rng.integers(1, 40))
        tap = int(rng.choice([0, 10]))
        a = spread_coeffs(n, x, k1, k2, nl, False, tap)
        b = O.spread_coeffs(n, x, k1, k2, nl, False, tap)
        assert a[0] == b[0]
        # the band-pass form differences two squared sincs (cancellation when
        # k1 ~ k2): FMA-contracted and plain evaluations differ by a few 1e-5
        scale = max(1e-30, float(np.abs(b[1]).max())) if len(b[1]) else 1.0
        np.testing.assert_allclose(a[1], b[1], rtol=2e-4, atol=2e-4 * scale)


def test_spread_coeffs_rejects_bad_band():
    L = _lib.lib()
    nl = C.c_int(10)
    off = C.c_int()
    buf = np.zeros(10, np.float32)
    assert L.rtm_spread_coeffs(100, 50.0, 0.4, 0.3, C.byref(nl), 0, 0, buf, C.byref(off)) == -1
    assert L.rtm_spread_coeffs(100, 150.0, 0.3, 0.4, C.byref(nl), 0, 0, buf, C.byref(off)) == -1


def test_create_rejects_bad_dims_without_gpu():
    L = _lib.lib()
    d = _lib.RtmDims(4, 4, 4, 10, 10, 10, 0.001)     # nx, nz < 9
    c = _lib.RtmConfig()
    L.rtm_config_default(C.byref(c))
    h = C.c_void_p()
    assert L.rtm_create(C.byref(d), C.byref(c), C.byref(h)) == -1
    assert not h.value
    assert b"out of range" in L.rtm_last_error(None)


def test_config_defaults_follow_reference():
    L = _lib.lib()
    c = _lib.RtmConfig()
    L.rtm_config_default(C.byref(c))
    assert (c.pml3d, c.top_pml, c.q_order) == (1, 1, 4)
    assert abs(c.pml_eps - 1e-3) < 1e-9 and abs(c.pml3d_scaler - 0.3) < 1e-7


@pytest.mark.parametrize("n", [20, 27, 64])
@pytest.mark.parametrize("isign", [1, -1])
def test_r2r_line_matrix_matches_oracle(n, isign):
    """The engine's FFTWR2R line matrix (built on the host, applied on the GPU
    as GEMMs) against the oracle's line derivative, column by column."""
    D = np.zeros(n * n, np.float32)
    assert _lib.lib().rtm_r2r_line_matrix(n, 10.0, isign, D) == 0
    D = D.reshape(n, n).astype(np.float64)
    want = np.stack([O.r2r_line(np.eye(n)[u], 10.0, isign) for u in range(n)], 1)
    assert np.abs(D - want).max() <= 1e-6 * np.abs(want).max()
    x = np.random.default_rng(n).standard_normal(n)
    np.testing.assert_allclose(D @ x, O.r2r_line(x, 10.0, isign), rtol=0, atol=1e-5 * np.abs(D @ x).max())
    assert _lib.lib().rtm_r2r_line_matrix(n, 10.0, 0, np.zeros(n * n, np.float32)) != 0
