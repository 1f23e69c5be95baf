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


def test_new_entry_points_validate_arguments_without_gpu():
    """Engines 0-6 only; the FK spreading and the learned-snapshot fallback
    refuse bad arguments before touching a device."""
    from konglong_b200.propagator import FkArgs
    L = _lib.lib()
    d = _lib.RtmDims(32, 32, 32, 10, 10, 10, 0.001)
    c = _lib.RtmConfig()
    L.rtm_config_default(C.byref(c))
    c.engine = 7
    h = C.c_void_p()
    assert L.rtm_create(C.byref(d), C.byref(c), C.byref(h)) == -1 and not h.value
    assert L.rtm_set_compressor_fallback(None, 1e-3, 0.1) == -1
    good = dict(nx=16, ny=8, nt=50, ntfft=64, dt=0.004, dx=10.0, dy=10.0, vsurf=1500.0, z=10.0, trueamp=1,
                deghost=1, side=-1, flcut=0.0, flpass=0.0, ghost_threshold=0.1, khpass=0.4, khcut=0.48, nlimit=20,
                domain=0, fmax=60.0)
    xy = np.array([[3.5, 2.0]], np.float32)
    tr = np.zeros((1, 50), np.float32)
    out = np.zeros((8, 16, 50), np.float32)
    bad = [dict(ntfft=40), dict(side=0), dict(khpass=0.5, khcut=0.4), dict(domain=2), dict(domain=1, nx=1),
           dict(domain=1, khpass=0.48), dict(ghost_threshold=0.0), dict(vsurf=0.0)]
    for b in bad:
        a = FkArgs(**{**good, **b})
        o = np.zeros((a.ny, a.nx, a.nt), np.float32)
        assert L.rtm_fk_spread(C.byref(a), 1, xy.ravel(), tr.ravel(), o.ravel()) == -1, b
    a = FkArgs(**good)
    for pos in ([[16.0, 2.0]], [[3.0, -0.5]], [[np.nan, 1.0]]):  # off the grid
        p = np.array(pos, np.float32)
        assert L.rtm_fk_spread(C.byref(a), 1, p.ravel(), tr.ravel(), out.ravel()) == -1, pos


def test_every_handle_entry_point_rejects_a_null_handle():
    """Every call that takes a handle (engine, batch or compressor) returns a
    negative status for a null one and touches nothing else - no device, no
    crash: the reference's assertion()/exit paths become status codes."""
    raw = C.CDLL(_lib.lib()._name)
    skip = {"rtm_config_default", "rtm_last_error", "rtm_ae_nparams", "rtm_spread_coeffs", "rtm_r2r_line_matrix",
            "rtm_fk_spread", "rtm_phase_correct", "rtm_c16_compress_noalloc", "rtm_create", "rtm_batch_create", "rtm_ae_create"}
    checked = 0
    for name in _lib.EXPORTS:
        typed = getattr(_lib.lib(), name)
        at = list(typed.argtypes or [])
        if name in skip or not at or at[0] is not C.c_void_p:
            continue
        f = getattr(raw, name)
        conv = [t if t in (C.c_int, C.c_float, C.c_double, C.c_longlong, C.c_size_t) else C.c_void_p for t in at]
        f.argtypes, f.restype = conv, C.c_int
        args = [0.0 if t in (C.c_float, C.c_double) else (None if t is C.c_void_p else 0) for t in conv]
        assert f(*args) < 0, name
        checked += 1
    assert checked >= 40


@pytest.mark.parametrize("bad", [dict(model_type=0), dict(model_type=4), dict(q_order=0), dict(q_order=9),
                                 dict(pml_eps=0.0), dict(pml_eps=1.0), dict(vmax=0.0), dict(engine=-1)])
def test_create_rejects_bad_configuration_without_gpu(bad):
    L = _lib.lib()
    d = _lib.RtmDims(32, 32, 32, 10, 10, 10, 0.001)
    c = _lib.RtmConfig()
    L.rtm_config_default(C.byref(c))
    for k, v in bad.items():
        setattr(c, k, v)
    h = C.c_void_p()
    assert L.rtm_create(C.byref(d), C.byref(c), C.byref(h)) == -1 and not h.value


def test_noalloc_codec_rejects_bad_arguments_without_gpu():
    L = _lib.lib()
    f = C.CDLL(L._name).rtm_c16_compress_noalloc
    f.argtypes, f.restype = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p], C.c_int
    assert f(None, None, 8, 8, 8, None) == -1
    assert f(C.c_void_p(16), C.c_void_p(32), 8, 0, 8, None) == -1
    assert f(C.c_void_p(16), C.c_void_p(32), 8, 1 << 20, 8, None) == -1  # more y slabs than the fixed scratch
    assert f(C.c_void_p(16), C.c_void_p(32), 1, 65536, 1, None) == -1    # one above RTM_NOALLOC_MAX_SLABS
