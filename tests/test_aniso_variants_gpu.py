"""FD8 VTI / TTI two-pass kernels against each other: 4 z cells per thread with
TMA rings (variant 3, the default when nz % 4 == 0 and the state is FP32) and one
cell per thread (variant 1) compute the same arithmetic in the same order, so the
modelling traces and wavefields are bit-equal - VTI and TTI, the Q update, both PML
modes, z faces a multiple of 4 cells wide and not, ragged tiles in x, y and z,
PML-free interior tiles next to PML tiles - and the 4-cell kernels match the CPU
oracle.  RTM images (fused snapshot store and imaging condition in the gradient
pass) are compared to 1e-5 (relative L2): the backward pass injects overlapping
receiver spread kernels with atomic adds, whose summation order varies."""
import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200.propagator import Propagator, spread_coeffs
from konglong_b200.spec import BACKWARD, ENGINE_FD8, FIELD_IMAGE, FIELD_W0, FIELD_W1, FORWARD, SNAP_C16, \
    SNAP_FP32, TTI, VTI, PropSpec
from oracle import pyoracle as O
from tests.conftest import rel_l2

pytestmark = pytest.mark.gpu


def _aniso_shot(nx, ny, nz, model, pml=8, use_q=False, pml3d=True, nt=60, seed=21):
    rng = np.random.default_rng(seed)
    spec = PropSpec(nx=nx, ny=ny, nz=nz, engine=ENGINE_FD8, model_type=model, use_q=use_q, nbnd=(pml,) * 6,
                    pml3d=pml3d, vmax=4500.0)
    sm = lambda: W.smooth_field(spec.shape, 2.0, rng)
    vel = np.clip(2500.0 * (1.0 + 0.3 * sm()), 1500.0, 4500.0).astype(np.float32)
    eps = W.minmax(sm(), 0.0, 0.2)
    dl = W.minmax(sm(), 0.0, 0.08)
    pjx = pjy = invq = None
    if model == TTI:
        theta = np.deg2rad(W.minmax(sm(), 0.0, 45.0))
        phi = np.deg2rad(W.minmax(sm(), 0.0, 360.0))
        pjx = (-np.sin(theta) * np.cos(phi)).astype(np.float32)
        pjy = (-np.sin(theta) * np.sin(phi)).astype(np.float32)
    if use_q:
        invq = (1.0 / W.minmax(sm(), 30.0, 200.0)).astype(np.float32)
    spec.dt = float(min(spec.dt, W.cfl_dt(spec, vel, eps, dl, pjx, pjy, invq, maxfreq=60.0)))
    src = (nx / 2 - 0.3, ny / 2 + 0.2, pml + 1.4)
    rx = np.linspace(1, nx - 2, 5)
    ry = np.linspace(0, ny - 1, 3)
    rxx, ryy = np.meshgrid(rx, ry, indexing="xy")
    rcv = np.stack([rxx.ravel(), ryy.ravel(), np.full(rxx.size, pml + 2.0)], 1).astype(np.float32)
    return W.Shot(spec, nt, vel, eps=eps, dl=dl, pjx=pjx, pjy=pjy, invq=invq,
                  wavelet=W.ricker(25.0, spec.dt, nt), src_pos=src, rcv_pos=rcv, interval=4, fpeak=25.0,
                  name="aniso_ragged")


def _engine(shot, variant, cls=Propagator):
    s = shot.spec
    s.kernel_variant = variant
    p = cls(s)
    if s.use_q:
        p.set_q_coeffs(*W.q_coefficients(s.dt, shot.fpeak))
    p.set_model(**shot.model_arrays())
    k1, k2 = W.spread_band(s)
    src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    rcv = W.make_traceset(shot.rcv_pos, s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    return p, src, rcv


def _modelling(shot, p, src, rcv):
    p.set_injection(src, shot.wavelet[None, :], shot.spec.dt_dxyz)
    p.set_extraction(rcv, shot.nt)
    p.reset()
    p.modelling(shot.nt, -1, 1)
    return p.traces(), p.get(FIELD_W1), p.get(FIELD_W0)


def _rtm(shot, p, src, rcv, fmt):
    nt = shot.nt
    rng = np.random.default_rng(5)
    data = (rng.standard_normal((rcv.ntr, nt)) * 1e3).astype(np.float32)
    p.snapshot_setup(fmt, (nt - 1) // shot.interval + 1)
    p.reset()
    p.set_injection(src, shot.wavelet[None, :], shot.spec.dt_dxyz)
    p.migration(FORWARD, 0, nt, -1, shot.interval)
    p.reset()
    p.image_setup(3, 4, 1)
    p.set_injection(rcv, data, shot.spec.dt_dxyz)
    p.migration(BACKWARD, nt - 1, -1, -1, shot.interval)
    return p.get(FIELD_IMAGE)


GRIDS = [
    # nx, ny, nz, model, pml, use_q, pml3d
    (44, 23, 52, VTI, 8, False, True),    # ragged x and z tiles, z faces a multiple of 4
    (37, 20, 44, TTI, 8, True, True),     # TTI + Q
    (50, 30, 64, VTI, 8, False, False),   # per-axis PML rounds (no cross terms)
    (41, 19, 48, TTI, 6, False, True),    # z faces of 6 cells: per-cell PML in the 4-cell kernels
    (70, 40, 100, TTI, 8, False, True),   # PML-free interior tiles next to PML tiles
]


@pytest.mark.parametrize("grid", GRIDS)
def test_variants_bit_equal(grid):
    nx, ny, nz, model, pml, use_q, pml3d = grid
    shot = _aniso_shot(nx, ny, nz, model, pml=pml, use_q=use_q, pml3d=pml3d)
    out = {}
    variants = (1, 3, 7, 0) if use_q else (1, 3, 0)
    for v in variants:
        p, src, rcv = _engine(shot, v)
        out[v] = _modelling(shot, p, src, rcv) + (_rtm(shot, p, src, rcv, SNAP_FP32), _rtm(shot, p, src, rcv, SNAP_C16))
        p.close()
    assert np.abs(out[1][0]).max() > 0 and np.abs(out[1][3]).max() > 0
    names = ("traces", "w1", "w0", "image fp32 snapshots", "image c16 snapshots")
    bad = []
    for v in variants[1:]:
        for k, (a, b) in enumerate(zip(out[1], out[v])):
            if k < 3 and not np.array_equal(a, b):
                bad.append(f"variant {v} {names[k]}: {int((a != b).sum())} cells differ")
            if k >= 3 and rel_l2(b, a) > 1e-5:
                bad.append(f"variant {v} {names[k]}: rel. L2 {rel_l2(b, a):.3g}")
    assert not bad, "; ".join(bad)


def test_autotuned_shapes_bit_equal():
    """Whatever the autotuner keeps (one-cell tile widths or 4-cell y segments) gives the same wavefields."""
    shot = _aniso_shot(60, 44, 96, TTI)
    p, src, rcv = _engine(shot, 1)
    ref = _modelling(shot, p, src, rcv)
    p.close()
    for steps in (1, 3):
        p, src, rcv = _engine(shot, 0)
        p.autotune(steps)
        assert any(r[0] == 4 for r in p.autotune_results())  # the 4-cell kernels were candidates
        got = _modelling(shot, p, src, rcv)
        p.close()
        for a, b in zip(ref, got):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("model,use_q", [(VTI, False), (TTI, True)])
def test_4cell_kernels_match_oracle(model, use_q):
    shot = _aniso_shot(44, 23, 52, model, use_q=use_q, nt=50)
    p, src, rcv = _engine(shot, 3)
    got = _modelling(shot, p, src, rcv)
    o, src, rcv = _engine(shot, 3, cls=O.Oracle)
    want = _modelling(shot, o, src, rcv)
    assert np.abs(want[0]).max() > 0
    assert rel_l2(got[0], want[0]) < 1e-4
    assert rel_l2(got[1], want[1]) < 1e-4


@pytest.mark.parametrize("q_bf16", [False, True])
def test_q_memory_ring_bit_equal(q_bf16):
    """The divergence pass's TMA ring carries the Q memory (FP32 or BF16) and 1/Q
    of its planes (variant 3 / 0); variant 7 keeps the update loading them
    itself and variant 1 is the one-cell pass: all compute the same bits,
    with ragged x / y / z tiles and PML tiles."""
    shot = _aniso_shot(45, 26, 56, TTI, use_q=True, nt=70)
    shot.spec.q_bf16 = q_bf16
    out = {}
    for v in (1, 7, 3, 0):
        p, src, rcv = _engine(shot, v)
        out[v] = _modelling(shot, p, src, rcv)
        p.close()
    assert np.abs(out[1][0]).max() > 0
    for v in (7, 3, 0):
        for k, name in enumerate(("traces", "w1", "w0")):
            np.testing.assert_array_equal(out[v][k], out[1][k], err_msg=f"variant {v} {name}")

