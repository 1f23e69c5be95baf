"""Parity with the reference's own CPU propagator at the full sizes of the
measured workloads.

The reference side is `oracle/_ref` (bgprtm's KernelCPU / FdEngine_fd /
FdEngine_cfd / PML compiled from its sources) driven by the restated loop of
Propagator::modelling (bgprtm/Propagator.cpp:1099-1153: kernel, update2nd,
Receiver::apply_src, extract_value, swap).  The CUDA path runs through the C
ABI on identical seeded models.  Bounds (relative L2):
  * FD8 receiver traces and wavefields: 1e-4 after 1000 steps, and every FD8
    operator step 2e-6 (FP32 rounding);
  * compact FD: within twice the reference's own FP32-vs-FP64 spread of the
    FP64 oracle (its band LU amplifies rounding);
the error of each result against the FP64 oracle is printed.
"""
import gc

import numpy as np
import pytest

from konglong_b200 import workloads as W
from konglong_b200.propagator import Propagator, spread_coeffs
from konglong_b200.spec import BACKWARD, FIELD_IMAGE, FIELD_W1, FORWARD, SNAP_FP32
from oracle import pyoracle as O
from tests.conftest import rel_l2

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")]


def _traces(shot, x, nts):
    s = shot.spec
    k1, k2 = W.spread_band(s)
    src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    rcv = W.make_traceset(shot.rcv_pos, s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    x.set_model(**{k: v for k, v in shot.model_arrays().items() if v is not None})
    x.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
    x.set_extraction(rcv, nts)
    x.reset()
    x.modelling(nts, -1, 1)
    return x.traces(), x.get(FIELD_W1 if isinstance(x, Propagator) else 1)


def test_iso128_full_shot_matches_reference():
    """128^3 ISO FD8, PML 20, 1000 steps, 64 x 64 receivers: traces and the
    final wavefield against the compiled KernelCPU."""
    shot = W.iso128(scale=1.0, nt=1000)
    got_tr, got_w = _traces(shot, Propagator(shot.spec), 1000)
    ref = O.Reference(shot.spec)
    ref_tr, ref_w = _traces(shot, ref, 1000)
    ref.close()
    d = O.Oracle(shot.spec, double=True)
    ex_tr, ex_w = _traces(shot, d, 1000)
    del d
    assert np.abs(ref_tr).max() > 0
    e_tr, e_w = rel_l2(got_tr, ref_tr), rel_l2(got_w, ref_w)
    print(f"iso128 1000 steps: traces {e_tr:.2e}, wavefield {e_w:.2e} vs reference; "
          f"vs FP64 oracle: GPU {rel_l2(got_tr, ex_tr):.2e} / {rel_l2(got_w, ex_w):.2e}, "
          f"reference {rel_l2(ref_tr, ex_tr):.2e} / {rel_l2(ref_w, ex_w):.2e}")
    assert e_tr < 1e-4
    assert e_w < 1e-4


def test_iso128_full_rtm_image_matches_oracle():
    """The 128^3 ISO RTM shot: 1000 forward steps with FP32 snapshots every 4
    steps, 1000 backward steps with the zero-lag imaging condition, against
    the FP32 oracle (the restated Propagator loop; the reference's migration
    loop does not compile) and, stated, the FP64 oracle."""
    shot = W.iso128(scale=1.0, nt=1000)
    s = shot.spec
    k1, k2 = W.spread_band(s)
    src = W.make_traceset([shot.src_pos], s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    rcv = W.make_traceset(shot.rcv_pos, s.nx, s.ny, s.nz, 10, k1, k2, spread_coeffs)
    data = (np.random.default_rng(17).standard_normal((rcv.ntr, 1000)) * 1e3).astype(np.float32)
    nt, interval = 1000, 4

    def rtm(x):
        x.set_model(vel=shot.vel)
        x.snapshot_setup(SNAP_FP32, (nt - 1) // interval + 1)
        x.reset()
        x.set_injection(src, shot.wavelet[None, :], s.dt_dxyz)
        x.migration(FORWARD, 0, nt, -1, interval)
        x.reset()
        x.image_setup(20, 10, 1)
        x.set_injection(rcv, data, s.dt_dxyz)
        x.migration(BACKWARD, nt - 1, -1, -1, interval)
        return x.get(FIELD_IMAGE if isinstance(x, Propagator) else 3)

    got = rtm(Propagator(s))
    o = O.Oracle(s)
    want = rtm(o)
    del o
    gc.collect()
    d = O.Oracle(s, double=True)
    exact = rtm(d)
    del d
    assert np.abs(want).max() > 0
    print(f"iso128 RTM image: {rel_l2(got, want):.2e} vs FP32 oracle, {rel_l2(got, exact):.2e} vs FP64 "
          f"(FP32 oracle vs FP64: {rel_l2(want, exact):.2e})")
    assert rel_l2(got, want) < 1e-4


def _operator_steps(x, model, w0, w1, steps, get=1):
    x.set_model(**model)
    x.put(0, w0)
    x.put(1, w1)
    for _ in range(steps):
        x.kernel()
        x.update2nd()
        x.swap()
    return x.get(get)


def _fields(shape, seed):
    rng = np.random.default_rng(seed)
    return W.smooth_field(shape, 2.0, rng), W.smooth_field(shape, 2.0, rng)


def test_vti_cfd_512x512x400_operator_steps_match_reference():
    """The full 512 x 512 x 400 VTI compact-FD grid (PML 32): three operator
    steps on smooth wavefields against the compiled KernelCPU (FdEngine_cfd)."""
    shot = W.vti_cfd(scale=1.0, nt=10)
    s = shot.spec
    model = dict(vel=shot.vel, eps=shot.eps, dl=shot.dl)
    w0, w1 = _fields(s.shape, 5)
    got = _operator_steps(Propagator(s), model, w0, w1, 3, FIELD_W1)
    gc.collect()
    r = O.Reference(s)
    ref = _operator_steps(r, model, w0, w1, 3)
    r.close()
    del r
    gc.collect()
    d = O.Oracle(s, double=True)
    exact = _operator_steps(d, model, w0, w1, 3)
    del d
    gc.collect()
    spread = rel_l2(ref, exact)
    print(f"vti_cfd 512x512x400 3 steps: GPU vs FP64 {rel_l2(got, exact):.2e}, reference vs FP64 {spread:.2e}, "
          f"GPU vs reference {rel_l2(got, ref):.2e}")
    assert np.abs(exact).max() > 0
    assert rel_l2(got, exact) < 2 * spread + 1e-6
    assert rel_l2(got, ref) < 3 * spread + 1e-6


def test_tti_640x640x512_operator_steps_match_reference():
    """The full 640 x 640 x 512 TTI grid (PML 32, FD8): three operator steps
    against the compiled KernelCPU (no Q: the reference harness restates the
    plain update2nd), then the same steps with the Q memory against the FP32
    oracle (Propagator::update2nd's Q branch restated)."""
    shot = W.tti_q(scale=1.0, nt=10)
    s = shot.spec
    model = dict(vel=shot.vel, eps=shot.eps, dl=shot.dl, pjx=shot.pjx, pjy=shot.pjy)
    w0, w1 = _fields(s.shape, 6)
    s.use_q = False
    got = _operator_steps(Propagator(s), model, w0, w1, 3, FIELD_W1)
    gc.collect()
    r = O.Reference(s)
    ref = _operator_steps(r, model, w0, w1, 3)
    r.close()
    del r
    gc.collect()
    print(f"tti 640x640x512 3 FD8 steps: GPU vs reference {rel_l2(got, ref):.2e}")
    assert np.abs(ref).max() > 0
    assert rel_l2(got, ref) < 2e-6
    del got, ref
    gc.collect()
    s.use_q = True
    cq0, cq, wq = W.q_coefficients(s.dt, shot.fpeak)
    model["invq"] = shot.invq
    g = Propagator(s)
    g.set_q_coeffs(cq0, cq, wq)
    got = _operator_steps(g, model, w0, w1, 3, FIELD_W1)
    del g
    gc.collect()
    o = O.Oracle(s)
    o.set_q_coeffs(cq0, cq, wq)
    want = _operator_steps(o, model, w0, w1, 3)
    del o
    print(f"tti+q 640x640x512 3 FD8 steps: GPU vs FP32 oracle {rel_l2(got, want):.2e}")
    assert rel_l2(got, want) < 2e-6
