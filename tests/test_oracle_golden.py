"""The oracle (CPU restatement) against the reference's own compiled kernels.

Fixtures come from oracle/_ref (bgprtm's KernelCPU / FdEngine_fd /
FdEngine_cfd / FdEngine_r2c / Cfd_plan / PML / WaveFieldCompress built from
source), see
tests/golden/make_golden.py.  FD8 must agree to FP32 rounding; the compact-FD
line solve (band LU without pivoting, pivots down to ~0.016) amplifies FP32
rounding, so its bound is the reference's own FP32-vs-FP64 spread.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests.conftest import rel_l2
from tests.golden_inputs import CASES, case_inputs, codec_input

FD8_TOL = 2e-6


def run_oracle(c, double=False):
    spec, model, w0, w1 = case_inputs(c)
    o = O.Oracle(spec, double=double)
    o.set_model(**model)
    o.put(0, w0)
    o.put(1, w1)
    for _ in range(c["steps"]):
        o.kernel()
        o.update2nd()
        o.swap()
    return o.get(1)


@pytest.mark.parametrize("name", [k for k in CASES if "fd8" in k])
def test_fd8_matches_reference(golden, name):
    got = run_oracle(CASES[name])
    ref = golden[f"{name}__w1"]
    assert rel_l2(got, ref) < FD8_TOL


@pytest.mark.parametrize("name", [k for k in CASES if "cfd" in k])
def test_cfd_matches_reference_within_fp32_conditioning(golden, name):
    got = run_oracle(CASES[name])
    exact = run_oracle(CASES[name], double=True)
    ref = golden[f"{name}__w1"]
    spread = rel_l2(ref, exact)           # the reference's own FP32 error
    assert spread < 5e-3
    assert rel_l2(got, ref) < 2.0 * spread + 1e-6
    assert rel_l2(got, exact) < 2.0 * spread + 1e-6


@pytest.mark.parametrize("name", [k for k in CASES if "r2c" in k or "r2r" in k])
def test_r2c_matches_reference(golden, name):
    """FFTWR2C / FFTWR2R: the reference's FdEngine_r2c / FdEngine_r2r (FFTW
    calls answered by their defining sums in double, Util::transpose
    completed) against the oracle's circulant / line-matrix forms."""
    got = run_oracle(CASES[name])
    assert rel_l2(got, golden[f"{name}__w1"]) < FD8_TOL
    assert rel_l2(run_oracle(CASES[name], double=True), golden[f"{name}__w1"]) < FD8_TOL


@pytest.mark.parametrize("n", [16, 17, 30, 27])
@pytest.mark.parametrize("isign", [1, -1])
def test_r2c_line_is_the_spectral_product(n, isign):
    """The oracle's circulant equals rfft -> i k_j (bin n/2 times isign) ->
    unnormalised irfft written with numpy's FFT, k_j = -j dk in float as
    FdEngine_r2c::assignW."""
    x = np.random.default_rng(n).standard_normal(n)
    sc = np.float32(1.0) / np.float32(n)
    dk = np.float32(2.0 * np.pi / np.float64(np.float32(10.0) * np.float32(n)) * np.float64(sc))
    k = np.array([np.float32(-j) * dk for j in range(n // 2 + 1)], np.float64)
    m = 1j * k
    m[n // 2] *= isign
    want = np.fft.irfft(np.fft.rfft(x) * m, n) * n
    np.testing.assert_allclose(O.r2c_line(x, 10.0, isign), want, rtol=0, atol=1e-12 * np.abs(want).max())


def test_r2c_known_answer_sine():
    """FdEngine_r2c's k_j = -j dk makes the engine's first derivative the
    negative of d/dx: sin(2 pi t / n) -> -(2 pi / (n d)) cos(2 pi t / n)."""
    n, d = 48, 10.0
    t = np.arange(n)
    got = O.r2c_line(np.sin(2 * np.pi * 3 * t / n), d, 1)
    want = -(2 * np.pi * 3 / (n * d)) * np.cos(2 * np.pi * 3 * t / n)
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-6 * np.abs(want).max())


def test_r2c_odd_lines_have_a_growing_mode():
    """The isign factor on bin n/2 (FdEngine_r2c.cpp:228-231) is +1 in the
    gradient pass and -1 in the divergence pass: for even n that bin is the
    Nyquist bin and drops out, for odd n it is an ordinary bin whose two-pass
    product is +k^2, a growing mode of the time stepping."""
    for n, grows in ((50, False), (51, True)):
        e = np.eye(n)
        dp = np.stack([O.r2c_line(e[i], 10.0, 1) for i in range(n)], 1)
        dm = np.stack([O.r2c_line(e[i], 10.0, -1) for i in range(n)], 1)
        top = np.linalg.eigvals(dm @ dp).real.max()
        assert (top > 1e-3) == grows, (n, top)


def test_r2r_is_stable_and_close_to_the_spectral_second_derivative():
    """FFTWR2R's two passes (DCT-II -> shifted bins -> DST-III, then DST-II ->
    DCT-III) make a non-positive operator for even and odd n whose low
    eigenvalues are -(pi m / (n d))^2 to high accuracy."""
    n, d = 40, 10.0
    for nn in (n, n + 1):
        e = np.eye(nn)
        dp = np.stack([O.r2r_line(e[i], d, 1) for i in range(nn)], 1)
        dm = np.stack([O.r2r_line(e[i], d, -1) for i in range(nn)], 1)
        ev = np.sort(np.linalg.eigvals(dm @ dp).real)[::-1]
        assert ev[0] < 1e-9
        m = np.arange(1, 6)
        np.testing.assert_allclose(-ev[1:6], (np.pi * m / (nn * d)) ** 2, rtol=1e-6)


def test_codec_bit_exact(golden):
    for cname, (a, nx, ny, nz) in codec_input().items():
        codes = O.c16_compress(a, nx, ny, nz)
        np.testing.assert_array_equal(codes, golden[f"c16_{cname}__codes"])
        dec = O.c16_uncompress(codes, nx, ny, nz).reshape(ny, nx, nz)
        ref = golden[f"c16_{cname}__decoded"].reshape(ny, nx, nz)
        # untapered cells decode bit-exactly; in the 20/10-cell edge tapers the
        # reference build (-ffast-math) may reassociate the taper products
        inner = (slice(20, -20) if ny > 40 else slice(None), slice(20, -20) if nx > 40 else slice(None),
                 slice(10, -10) if nz > 20 else slice(None))
        np.testing.assert_array_equal(dec[inner].view(np.uint32), ref[inner].view(np.uint32))
        np.testing.assert_allclose(dec, ref, rtol=1e-6, atol=0)


@pytest.mark.parametrize("n", [40, 57])
@pytest.mark.parametrize("s", [0, 1])
def test_cfd_plan(golden, n, s):
    bm, bl, am = O.cfd_plan(n, 10.0, s)
    np.testing.assert_array_equal(bm, golden[f"cfd_plan_{n}_{s}__bm"])
    np.testing.assert_array_equal(bl, golden[f"cfd_plan_{n}_{s}__bl"])
    np.testing.assert_allclose(am, golden[f"cfd_plan_{n}_{s}__am"], rtol=1e-6, atol=0)


def test_taylor_weights_order8():
    c1, c2 = O.taylor_weights(4)
    np.testing.assert_allclose(c1[1:], [4 / 5, -1 / 5, 4 / 105, -1 / 280], rtol=1e-13)
    np.testing.assert_allclose(c2, [-205 / 72, 8 / 5, -1 / 5, 8 / 315, -1 / 560], rtol=1e-13)


def test_fd8_known_answer_sine():
    """FdEngine::init_sine-style field (bgprtm/FdEngine.cpp:404-421): the FD8
    Laplacian of sin(kx x) sin(kz z) sin(ky y) is -(kx^2+ky^2+kz^2) times the
    field, up to the FD8 dispersion at these wavenumbers."""
    from konglong_b200.spec import PropSpec
    nx, ny, nz = 40, 36, 44
    spec = PropSpec(nx=nx, ny=ny, nz=nz, dx=10, dy=10, dz=10, dt=0.001, nbnd=(0,) * 6)
    kx, ky, kz = 2 * np.pi / 20, 2 * np.pi / 18, 2 * np.pi / 22   # per cell
    iy, ix, iz = np.meshgrid(np.arange(ny), np.arange(nx), np.arange(nz), indexing="ij")
    f = (np.sin(kx * ix) * np.sin(ky * iy) * np.sin(kz * iz)).astype(np.float32)
    o = O.Oracle(spec, double=True)
    vel = np.full(spec.shape, 1.0 / spec.dt, np.float32)   # (v dt)^2 = 1
    o.set_model(vel=vel)
    o.put(1, f)
    o.put(0, np.zeros_like(f))
    o.kernel()
    lap = -o.get(0).reshape(spec.shape)
    interior = (slice(4, -4),) * 3
    want = -(kx ** 2 + ky ** 2 + kz ** 2) / 100.0 * f
    assert rel_l2(lap[interior], want[interior]) < 2e-4


def test_pml_profile(golden):
    # restated profile (float) against the reference's PML object
    from konglong_b200.spec import PropSpec
    w, d, dt, vmax = 20, 10.0, 0.001, 4500.0
    beta = np.float32(d) / (np.float32(dt) * np.float32(vmax))
    dg1 = np.float32(np.log(np.float32(1) / np.float32(1e-3))) / (np.float32(w) * beta)
    t = (np.float32(w) - np.arange(w, dtype=np.float32)) / np.float32(w)
    coef = np.float32(0.75) * t * t * dg1
    np.testing.assert_allclose(coef, golden["pml_coef_20"], rtol=1e-6)


@pytest.mark.parametrize("model", [1, 2])
def test_cfd_batch_is_the_compact_fd_path_without_cross_damping(model):
    """Engine CFD_BATCH (the Derivative path: Derivative_cfd + Boundary) and
    Engine CFD (KernelCPU + FdEngine_cfd) with pml3d off differ for ISO and
    VTI only in the order of the divergence sum, so in float64 they agree to
    rounding; for TTI the divergence pass takes plan 1 (iswitch) instead of 2."""
    from konglong_b200.spec import ENGINE_CFD, ENGINE_CFDB
    from tests.golden_inputs import case_inputs

    def run(engine, model, double):
        c = dict(engine=engine, model=model, shape=(24, 20, 28), pml=6, steps=3, seed=31, pml3d=False)
        spec, m, w0, w1 = case_inputs(c)
        o = O.Oracle(spec, double=double)
        o.set_model(**m)
        o.put(0, w0)
        o.put(1, w1)
        for _ in range(3):
            o.kernel()
            o.update2nd()
            o.swap()
        return o.get(1)

    assert rel_l2(run(ENGINE_CFDB, model, True), run(ENGINE_CFD, model, True)) < 1e-11
    assert rel_l2(run(ENGINE_CFDB, 3, True), run(ENGINE_CFD, 3, True)) > 1e-3


def test_spread_coeffs_match_reference(golden):
    """The restated CompactOrmsbySpreadCoeff against the reference's own
    Util.cpp:317-397 (its libCommon sinc / dipole / Blackman from the
    stand-ins): same offsets and lengths; values to 1e-5 of the kernel's peak,
    plus the conditioning of the Ormsby difference (a2^2 sinc2^2 - a1^2 sinc1^2)
    / (a2 - a1) for nearly equal bands, where the reference's -ffast-math
    rounding differs."""
    from tests.golden_inputs import spread_cases
    offs, coefs = golden["spread_offsets"], golden["spread_coeffs"]
    for j, (n, x, k1, k2, nl, dip) in enumerate(spread_cases()):
        o, c = O.spread_coeffs(n, x, k1, k2, nl, dip, 0)
        assert (o, len(c)) == tuple(offs[j]), (j, n, x, nl)
        if len(c) == 0:  # x within half a cell of the edge: an empty kernel on both sides
            continue
        ref = coefs[j][:len(c)]
        tol = 1e-5 + (1e-7 / max(k2 - k1, 1e-6) if k1 != k2 and not dip else 0.0)
        assert np.abs(c - ref).max() <= tol * max(np.abs(ref).max(), 1e-30), (j, k2 - k1)


def test_iso_traces_match_the_homogeneous_green_function():
    """Known answer for the whole ISO chain (injection scaling, Vel2, FD8
    Laplacian, leapfrog, extraction): in a homogeneous medium the modelled
    receiver trace is the injected wavelet delayed by r / v over 4 pi r, the
    3-D acoustic Green's function (w_tt = v^2 lap w + v^2 s delta: the injection
    adds s (v dt)^2 k / (dx dy dz))."""
    from konglong_b200 import workloads as W
    from konglong_b200.spec import ENGINE_FD8, PropSpec
    n, pml, v, d, dt, nt = 72, 12, 2000.0, 10.0, 0.001, 260
    spec = PropSpec(nx=n, ny=n, nz=n, dx=d, dy=d, dz=d, dt=dt, engine=ENGINE_FD8, model_type=1, nbnd=(pml,) * 6,
                    vmax=v)
    wav = W.ricker(12.0, dt, nt)
    c = n // 2
    rs = (12.0, 18.0)
    k1, k2 = W.spread_band(spec)
    src = W.make_traceset([(c, c, c)], n, n, n, 10, k1, k2, O.spread_coeffs)
    rcv = W.make_traceset([(c + r, c, c) for r in rs], n, n, n, 10, k1, k2, O.spread_coeffs)
    o = O.Oracle(spec, double=True)
    o.set_model(vel=np.full(spec.shape, v, np.float32))
    o.set_injection(src, wav[None, :], spec.dt_dxyz)
    o.set_extraction(rcv, nt)
    o.reset()
    o.modelling(nt, -1, 1)
    tr = o.traces()
    t = np.arange(nt) * dt
    for j, (r, tol) in enumerate(zip(rs, (0.01, 0.02))):
        want = np.interp(t - r * d / v, t, wav, left=0, right=0) / (4 * np.pi * r * d)
        cc = tr[j] @ want / np.linalg.norm(tr[j]) / np.linalg.norm(want)
        amp = (tr[j] @ want) / (want @ want)
        assert cc > 0.998 and abs(amp - 1) < tol, (r, cc, amp)


@pytest.mark.parametrize("engine", [1, 2, 3, 4, 5, 6])
def test_first_derivative_engines_match_the_homogeneous_green_function(engine):
    """The two-pass first-derivative engines (compact FD, FFTWR2C, FFTWR2R,
    CFD_BATCH, FFTV, SINCOS; ISO) against the same 3-D Green's function: the
    engines' derivative conventions (FFTWR2C's k = -j dk makes each pass
    -d/dx) and boundary closures leave the propagating pulse exact to 0.1 %
    here.  For FFTV and SINCOS, whose libfftv filters the reference tree does
    not hold, this known answer is the pin."""
    from konglong_b200 import workloads as W
    from konglong_b200.spec import PropSpec
    n, pml, v, d, dt, nt = 64, 12, 2000.0, 10.0, 0.0008, 260
    spec = PropSpec(nx=n, ny=n, nz=n, dx=d, dy=d, dz=d, dt=dt, engine=engine, model_type=1, nbnd=(pml,) * 6, vmax=v)
    wav = W.ricker(12.0, dt, nt)
    c = n // 2
    k1, k2 = W.spread_band(spec)
    src = W.make_traceset([(c, c, c)], n, n, n, 10, k1, k2, O.spread_coeffs)
    rcv = W.make_traceset([(c + 12.0, c, c)], n, n, n, 10, k1, k2, O.spread_coeffs)
    o = O.Oracle(spec, double=True)
    o.set_model(vel=np.full(spec.shape, v, np.float32))
    o.set_injection(src, wav[None, :], spec.dt_dxyz)
    o.set_extraction(rcv, nt)
    o.reset()
    o.modelling(nt, -1, 1)
    tr = o.traces()[0]
    t = np.arange(nt) * dt
    want = np.interp(t - 120.0 / v, t, wav, left=0, right=0) / (4 * np.pi * 120.0)
    cc = tr @ want / np.linalg.norm(tr) / np.linalg.norm(want)
    amp = (tr @ want) / (want @ want)
    assert cc > 0.9995 and abs(amp - 1) < 0.005, (cc, amp)


@pytest.mark.parametrize("name", [k for k in CASES if k.endswith("_rho")])
def test_density_changes_the_reference_result(golden, name):
    """The density fixtures carry the density: the same step without it (rho
    = 1, ISO FD8 then on its Laplacian path) is far from the reference's."""
    c = dict(CASES[name])
    spec, model, w0, w1 = case_inputs(c)
    spec.use_rho = False
    model.pop("rho")
    o = O.Oracle(spec)
    o.set_model(**model)
    o.put(0, w0)
    o.put(1, w1)
    for _ in range(c["steps"]):
        o.kernel()
        o.update2nd()
        o.swap()
    assert rel_l2(o.get(1), golden[f"{name}__w1"]) > 1e-2


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference not built")
def test_reference_compact_fd_tti_grows_in_a_tilted_medium():
    """Recorded behaviour of the reference: its compact-FD TTI step (KernelCPU
    + FdEngine_cfd, compiled) grows without bound in a homogeneous medium with
    a 30-degree tilt, while its FD8 TTI step on the same model stays bounded;
    the oracle follows the compact-FD growth.  Long compact-FD runs are
    therefore compared on untilted TTI models."""
    from konglong_b200 import workloads as W
    from konglong_b200.propagator import spread_coeffs
    from konglong_b200.spec import ENGINE_CFD, ENGINE_FD8, TTI, PropSpec
    th, ph = np.deg2rad(30.0), np.deg2rad(45.0)
    peak = {}
    for eng in (ENGINE_CFD, ENGINE_FD8):
        s = PropSpec(nx=52, ny=52, nz=40, engine=eng, model_type=TTI, nbnd=(6,) * 6, vmax=4500.0, dt=0.0005)
        sh = s.shape
        m = dict(vel=np.full(sh, 3000, np.float32), eps=np.full(sh, 0.2, np.float32), dl=np.full(sh, 0.1, np.float32),
                 pjx=np.full(sh, -np.sin(th) * np.cos(ph), np.float32),
                 pjy=np.full(sh, -np.sin(th) * np.sin(ph), np.float32))
        k1, k2 = W.spread_band(s)
        src = W.make_traceset([(26, 26, 20)], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
        r = O.Reference(s, nthreads=4)
        r.set_model(**m)
        r.set_injection(src, W.ricker(20.0, s.dt, 30)[None, :], s.dt_dxyz)
        r.reset()
        r.run(0, 30)
        peak[eng] = float(np.abs(r.get(1)).max())
        r.close()
    assert peak[ENGINE_CFD] > 1e6
    assert peak[ENGINE_FD8] < 1e3


def test_fftv_odd_lines_are_stable():
    """FFTV's plain spectral derivative has no growing mode on odd lines (the
    FFTWR2C isign bin has one, test_r2c_odd_lines_have_a_growing_mode): the
    two passes multiply every bin by -k^2 <= 0."""
    from konglong_b200.spec import PropSpec
    for n in (23, 24):
        x = np.random.default_rng(n).standard_normal(n)
        y = O.r2c_line(O.r2c_line(x, 10.0, 1), 10.0, 1)
        # the composite operator is symmetric negative semi-definite: <x, D D x> <= 0
        assert x @ y <= 1e-9 * np.abs(x @ x)
    spec = PropSpec(nx=23, ny=21, nz=27, engine=5, model_type=1, nbnd=(4,) * 6, vmax=3000.0, dt=0.0008)
    o = O.Oracle(spec, double=True)
    o.set_model(vel=np.full(spec.shape, 3000.0, np.float32))
    w = np.random.default_rng(3).standard_normal(spec.shape).astype(np.float32)
    o.put(0, w)
    o.put(1, w)
    peak0 = float(np.abs(w).max())
    for _ in range(200):
        o.kernel()
        o.update2nd()
        o.swap()
    assert float(np.abs(o.get(1)).max()) < 10 * peak0
