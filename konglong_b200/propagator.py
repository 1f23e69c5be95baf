"""Host-side mirror of bgprtm's propagation interface over the CUDA engine.

`Propagator` exposes, on one GPU-resident shot, the operations the reference
splits across KernelCPU (bgprtm/KernelCPU.h:16-64), Propagator
(bgprtm/Propagator.h:100-148), Receiver / ExtractReceiverData and
WaveFieldCompress / ImagingCondition, with the reference's names and argument
meaning.  Every call goes through the C ABI of include/rtm_b200.h; errors
raise `RtmError` with the engine's message.  There is no CPU code path.
"""
import ctypes as C

import numpy as np

from . import _lib
from .spec import (FIELD_IMAGE, FIELD_W0, FORWARD, PropSpec, TraceSet)


def _arr(a, dtype=np.float32):
    return None if a is None else np.ascontiguousarray(a, dtype=dtype).ravel()


class Propagator:
    """One shot's wavefield state on the current CUDA device."""

    def __init__(self, spec: PropSpec):
        L = _lib.lib()
        self.L = L
        self.spec = spec
        d = _lib.RtmDims(spec.nx, spec.ny, spec.nz, spec.dx, spec.dy, spec.dz, spec.dt)
        c = _lib.RtmConfig()
        L.rtm_config_default(C.byref(c))
        c.engine, c.model_type = spec.engine, spec.model_type
        c.use_q, c.q_order = int(spec.use_q), spec.q_order
        for k in range(6):
            c.nbnd[k] = int(spec.nbnd[k])
        c.vmax, c.pml_eps = spec.vmax, spec.pml_eps
        c.pml3d, c.pml3d_scaler, c.top_pml = int(spec.pml3d), spec.pml3d_scaler, int(spec.top_pml)
        c.state_fp16 = int(spec.state_fp16)
        c.use_rho = int(getattr(spec, "use_rho", False))
        c.q_bf16 = int(getattr(spec, "q_bf16", False))
        c.kernel_variant = int(getattr(spec, "kernel_variant", 0))
        h = C.c_void_p()
        _lib.check(L.rtm_create(C.byref(d), C.byref(c), C.byref(h)), "rtm_create")
        self.h = h
        self.n = spec.n
        self._ext = None

    # -- lifetime -----------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.L.rtm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _ck(self, code, what):
        _lib.check(code, what, self.h)

    # -- model (KernelCPU::setModel + Propagator::Vel2, Q::updateCq) ----------------
    def set_q_coeffs(self, cq0, cq, wq):
        self._ck(self.L.rtm_set_q_coeffs(self.h, float(cq0), _arr(cq), _arr(wq)), "rtm_set_q_coeffs")

    def set_model(self, vel, eps=None, dl=None, pjx=None, pjy=None, invq=None, rho=None):
        """KernelCPU::setModel(vel, rho, del, eps, pjx, pjy) + Vel2; rho with spec.use_rho."""
        arrs = [_arr(a) for a in (vel, rho, eps, dl, pjx, pjy, invq)]
        for a in arrs:
            if a is not None and a.size != self.n:
                raise ValueError("model volume size does not match the grid")
        ptrs = [None if a is None else a.ctypes.data for a in arrs]
        self._ck(self.L.rtm_set_model(self.h, *ptrs), "rtm_set_model")

    # -- one step's pieces ----------------------------------------------------------
    def reset(self):
        self._ck(self.L.rtm_reset(self.h), "rtm_reset")

    def kernel(self):
        """KernelCPU::ISO / VTI / TTI: w0 -= (v dt)^2 L[w1] with PML."""
        self._ck(self.L.rtm_kernel(self.h), "rtm_kernel")

    def update2nd(self):
        self._ck(self.L.rtm_update2nd(self.h), "rtm_update2nd")

    def swap(self):
        self._ck(self.L.rtm_swap(self.h), "rtm_swap")

    # -- sources / receivers (Receiver::apply, ExtractReceiverData::extract) ---------
    def set_injection(self, ts: TraceSet, traces, scaler):
        tr = np.ascontiguousarray(traces, np.float32)
        self._ck(self.L.rtm_set_injection(self.h, ts.ntr, ts.lx, ts.ly, ts.lz, _arr(ts.off, np.int32),
                                          _arr(ts.len, np.int32), _arr(ts.kx), _arr(ts.ky), _arr(ts.kz),
                                          tr.ravel(), tr.shape[1], float(scaler)), "rtm_set_injection")

    def set_extraction(self, ts: TraceSet, nt_out):
        self._ext = (ts.ntr, nt_out)
        self._ck(self.L.rtm_set_extraction(self.h, ts.ntr, ts.lx, ts.ly, ts.lz, _arr(ts.off, np.int32),
                                           _arr(ts.len, np.int32), _arr(ts.kx), _arr(ts.ky), _arr(ts.kz),
                                           nt_out), "rtm_set_extraction")

    def inject(self, it):
        self._ck(self.L.rtm_inject(self.h, it), "rtm_inject")

    def extract(self, jt):
        self._ck(self.L.rtm_extract(self.h, jt), "rtm_extract")

    def traces(self):
        ntr, nt = self._ext
        out = np.zeros((ntr, nt), np.float32)
        self._ck(self.L.rtm_get_traces(self.h, out.ravel()), "rtm_get_traces")
        return out

    # -- snapshots and imaging --------------------------------------------------------
    def snapshot_setup(self, fmt, nslots):
        self._ck(self.L.rtm_snapshot_setup(self.h, fmt, nslots), "rtm_snapshot_setup")

    def snapshot_store(self, slot):
        self._ck(self.L.rtm_snapshot_store(self.h, slot), "rtm_snapshot_store")

    def snapshot_load(self, slot):
        out = np.zeros(self.n, np.float32)
        self._ck(self.L.rtm_snapshot_load(self.h, slot, out), "rtm_snapshot_load")
        return out

    def image_setup(self, ntaper_t=0, ntaper_z=0, edge=1):
        self._ck(self.L.rtm_image_setup(self.h, ntaper_t, ntaper_z, edge), "rtm_image_setup")

    def image_accumulate(self, slot):
        self._ck(self.L.rtm_image_accumulate(self.h, slot), "rtm_image_accumulate")

    # -- time loops (Propagator::modelling / migration) -------------------------------
    def modelling(self, nts, it_shift=-1, ntratio=1):
        self._ck(self.L.rtm_modelling(self.h, nts, it_shift, ntratio), "rtm_modelling")

    def migration(self, direction, it_begin, it_end, it_shift=-1, interval=1):
        self._ck(self.L.rtm_migration(self.h, direction, it_begin, it_end, it_shift, interval),
                 "rtm_migration")

    @property
    def last_loop_ms(self):
        v = C.c_float()
        self._ck(self.L.rtm_last_loop_ms(self.h, C.byref(v)), "rtm_last_loop_ms")
        return v.value

    def autotune(self, steps=5):
        """Pick the fastest launch shape for this grid (clobbers the state)."""
        ch = C.c_int(0)
        self._ck(self.L.rtm_autotune(self.h, steps, C.byref(ch)), "rtm_autotune")
        return ch.value

    def set_compressor_fallback(self, tau=1e-3, max_fraction=0.1):
        """Keep the high-energy blocks of learned snapshots as FP16 (max_fraction 0: off)."""
        self._ck(self.L.rtm_set_compressor_fallback(self.h, float(tau), float(max_fraction)),
                 "rtm_set_compressor_fallback")

    def image_condition(self, option):
        """spec.IC_IMAGE1 (zero-lag, default) or spec.IC_INVERSION (k-domain derivative terms)."""
        self._ck(self.L.rtm_image_condition(self.h, int(option)), "rtm_image_condition")

    def image_double(self, ndbl_z=2, ndbl_x=2, ndbl_y=2, high_z=0.9, high_xy=0.7):
        """Double-grid IMAGE1: the imaging condition on the grid doubled along z (and x, y),
        from half-shifted copies of both high-cut fields; (1, 1, 1) turns it off."""
        self._ck(self.L.rtm_image_double(self.h, int(ndbl_z), int(ndbl_x), int(ndbl_y), float(high_z),
                                         float(high_xy)), "rtm_image_double")
        self._dbl = (int(ndbl_y), int(ndbl_x), int(ndbl_z))

    def _get_double(self, fn, what):
        dy, dx, dz = self._dbl
        s = self.spec
        out = np.empty((s.ny * dy, s.nx * dx, s.nz * dz), np.float32)
        self._ck(fn(self.h, out.ctypes.data), what)
        return out

    def get_image_double(self):
        """The double-grid image, shape (ny * ndbl_y, nx * ndbl_x, nz * ndbl_z)."""
        return self._get_double(self.L.rtm_get_image_double, "rtm_get_image_double")

    def get_illum_double(self):
        """The source illumination interpolated onto the doubled grid."""
        return self._get_double(self.L.rtm_get_illum_double, "rtm_get_illum_double")

    def illum_setup(self, on=True):
        """Accumulate the source illumination (sum of squared source values) in the imaging condition."""
        self._ck(self.L.rtm_illum_setup(self.h, int(bool(on))), "rtm_illum_setup")

    def illum_compensate(self, smooth_xy=10, smooth_z=10, amp_damping=1.0, damp_weight=0.07):
        """Shot illumination compensation of the image (reference defaults)."""
        self._ck(self.L.rtm_illum_compensate(self.h, smooth_xy, smooth_z, amp_damping, damp_weight),
                 "rtm_illum_compensate")

    def snapshot_slot_bytes(self, fmt):
        b = C.c_size_t(0)
        self._ck(self.L.rtm_snapshot_slot_bytes(self.h, int(fmt), C.byref(b)), "rtm_snapshot_slot_bytes")
        return int(b.value)

    def snapshot_window(self, first):
        self._ck(self.L.rtm_snapshot_window(self.h, int(first)), "rtm_snapshot_window")

    def checkpoint_setup(self, nckpt):
        """Allocates nckpt checkpoint slots; returns the bytes of one slot."""
        b = C.c_size_t(0)
        self._ck(self.L.rtm_checkpoint_setup(self.h, int(nckpt), C.byref(b)), "rtm_checkpoint_setup")
        return int(b.value)

    def checkpoint_save(self, k):
        self._ck(self.L.rtm_checkpoint_save(self.h, int(k)), "rtm_checkpoint_save")

    def checkpoint_load(self, k):
        self._ck(self.L.rtm_checkpoint_load(self.h, int(k)), "rtm_checkpoint_load")

    def snapshot_offload(self, nstage):
        """Keep the snapshot slots in pinned host memory with `nstage` device staging slots (0: device slots)."""
        self._ck(self.L.rtm_snapshot_offload(self.h, int(nstage)), "rtm_snapshot_offload")

    def autotune_results(self):
        """[(family, shape, yseg, cfd_xy, ms)] of the candidates the last autotune timed."""
        out, k = [], 0
        desc, ms = (C.c_int * 4)(), C.c_float(0)
        while self.L.rtm_autotune_result(self.h, k, desc, C.byref(ms)) == 0:
            out.append((*desc, ms.value))
            k += 1
        return out

    def set_compressor(self, ae):
        """Attach a compressor.AutoEncoder for RTM_SNAP_AE snapshots (None detaches)."""
        self._ck(self.L.rtm_set_compressor(self.h, ae.a if ae is not None else None), "rtm_set_compressor")
        self._ae = ae  # keep it alive while attached

    def check_finite(self, field):
        """True when `field` (W0 / W1 / IMAGE) holds only finite values."""
        nf = C.c_int(0)
        self._ck(self.L.rtm_check_finite(self.h, field, C.byref(nf)), "rtm_check_finite")
        return nf.value == 0

    def selftest_bounded_wait(self):
        """Status code of the bounded-wait self-test (RTM_ERR_TIMEOUT when the
        engine's device waits give up as designed)."""
        return self.L.rtm_selftest_bounded_wait(self.h)

    def launch_count(self):
        v = C.c_longlong()
        self._ck(self.L.rtm_last_loop_launches(self.h, C.byref(v)), "rtm_last_loop_launches")
        return v.value

    def profile(self, on=True):
        self._ck(self.L.rtm_profile(self.h, int(on)), "rtm_profile")

    def profile_read(self):
        """{kernel kind: (total device ms, launches)} of the profiled loops."""
        ms = np.zeros(len(_lib.KERNEL_KINDS), np.float64)
        cnt = np.zeros(len(_lib.KERNEL_KINDS), np.int64)
        self._ck(self.L.rtm_profile_read(self.h, ms, cnt), "rtm_profile_read")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_lib.KERNEL_KINDS) if cnt[i]}

    # -- field access -------------------------------------------------------------------
    def get(self, field):
        out = np.zeros(self.n, np.float32)
        self._ck(self.L.rtm_get(self.h, field, out.ctypes.data), "rtm_get")
        return out

    def put(self, field, a):
        a = _arr(a)
        self._ck(self.L.rtm_put(self.h, field, a.ctypes.data), "rtm_put")

    # -- whole-shot drivers ----------------------------------------------------------
    def rtm_shot(self, src: TraceSet, src_traces, rcv: TraceSet, rcv_traces, nt, nts_fwd, interval,
                 snap_fmt=0, ntaper_t=0, ntaper_z=0, edge=1, it_shift=-1):
        """Propagator::rtm for one shot (bgprtm/Propagator.cpp:2157-2280): forward
        pass storing snapshots, backward pass with the zero-lag imaging condition
        fused into the step, image returned."""
        nslots = (nts_fwd - 1) // interval + 1
        self.snapshot_setup(snap_fmt, nslots)
        self.reset()
        self.set_injection(src, src_traces, self.spec.dt_dxyz)
        self.migration(FORWARD, 0, nts_fwd, it_shift, interval)
        fwd_ms = self.last_loop_ms
        self.reset()
        self.image_setup(ntaper_t, ntaper_z, edge)
        self.set_injection(rcv, rcv_traces, self.spec.dt_dxyz)
        self.migration(1, nt - 1, -1, it_shift, interval)
        bwd_ms = self.last_loop_ms
        return self.get(FIELD_IMAGE), fwd_ms, bwd_ms

    def rtm_shot_checkpointed(self, src: TraceSet, src_traces, rcv: TraceSet, rcv_traces, nt, nts_fwd, interval,
                              seg_slots, snap_fmt=0, ntaper_t=0, ntaper_z=0, edge=1, it_shift=-1):
        """Propagator::rtm for one shot whose snapshots do not all fit: store /
        recompute.  The snapshot slots hold seg_slots snapshots (one segment of
        seg_slots * interval steps).  The forward pass saves a checkpoint of the
        propagation state at the start of every segment but the last and
        stores the last segment's snapshots; the backward pass images the last
        segment, then for each earlier segment saves the receiver state,
        reloads the segment's source checkpoint, recomputes its snapshots,
        restores the receiver state and images the segment.  The result equals
        rtm_shot's (same arithmetic per step; the backward receiver injection's
        atomic adds may order differently).  Returns the image and the device
        ms of the forward, recompute and backward loops."""
        seg = checkpoint_plan(nts_fwd, interval, seg_slots)
        nseg = len(seg)
        self.snapshot_setup(snap_fmt, seg_slots)
        # checkpoint slots 0 .. nseg-2: the source segments; nseg-1: the receiver state
        self.checkpoint_setup(nseg if nseg > 1 else 0)
        self.reset()
        self.set_injection(src, src_traces, self.spec.dt_dxyz)
        self.snapshot_window(seg[-1][0] // interval)
        ms = {"forward": 0.0, "recompute": 0.0, "backward": 0.0}
        for j, (a, b) in enumerate(seg):
            if j < nseg - 1:
                self.checkpoint_save(j)
            self.migration(FORWARD, a, b, it_shift, interval)
            ms["forward"] += self.last_loop_ms
        self.reset()
        self.image_setup(ntaper_t, ntaper_z, edge)
        self.set_injection(rcv, rcv_traces, self.spec.dt_dxyz)
        hi = nt - 1
        for j in range(nseg - 1, -1, -1):
            a, b = seg[j]
            if j < nseg - 1:
                self.checkpoint_save(nseg - 1)
                self.checkpoint_load(j)
                self.snapshot_window(a // interval)
                self.set_injection(src, src_traces, self.spec.dt_dxyz)
                self.migration(FORWARD, a, b, it_shift, interval)
                ms["recompute"] += self.last_loop_ms
                self.checkpoint_load(nseg - 1)
                self.set_injection(rcv, rcv_traces, self.spec.dt_dxyz)
            self.migration(1, hi, a - 1, it_shift, interval)
            ms["backward"] += self.last_loop_ms
            hi = a - 1
        return self.get(FIELD_IMAGE), ms


def checkpoint_plan(nts_fwd, interval, seg_slots):
    """Segments [a, b) of the forward steps [0, nts_fwd) for store / recompute:
    each holds seg_slots snapshots (seg_slots * interval steps), the last one
    the remainder."""
    if interval < 1 or seg_slots < 1 or nts_fwd < 1:
        raise ValueError("checkpoint_plan: interval, seg_slots and nts_fwd must be positive")
    step = seg_slots * interval
    return [(a, min(a + step, nts_fwd)) for a in range(0, nts_fwd, step)]


def checkpoint_slots_for_budget(nts_fwd, interval, slot_bytes, ckpt_bytes, budget_bytes):
    """The largest segment (in snapshots) whose slots plus one checkpoint per
    segment (and one for the receiver state) fit budget_bytes; 0 when none
    does.  All snapshots fit when the return value covers nts_fwd."""
    nsnap = (nts_fwd - 1) // interval + 1
    for s in range(nsnap, 0, -1):
        nseg = -(-nsnap // s)
        if s * slot_bytes + (nseg if nseg > 1 else 0) * ckpt_bytes <= budget_bytes:
            return s
    return 0


class Batch:
    """Several ISO FD8 shots stepped together (rtm_batch_*): one persistent
    kernel per time step over every active shot's tiles, batched injection and
    extraction, the time loop as CUDA graphs.  The shots keep their own state:
    after `modelling`, each Propagator holds what its own `modelling` call
    would have produced."""

    def __init__(self, shots):
        self.L = _lib.lib()
        self.shots = list(shots)
        arr = (C.c_void_p * len(self.shots))(*[p.h for p in self.shots])
        b = C.c_void_p()
        _lib.check(self.L.rtm_batch_create(arr, len(self.shots), C.byref(b)), "rtm_batch_create")
        self.b = b

    def close(self):
        if getattr(self, "b", None):
            self.L.rtm_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def autotune(self, steps=5):
        """Fastest tile shape of the batched kernel (zeroes the shots' state)."""
        ch = C.c_int(0)
        _lib.check(self.L.rtm_batch_autotune(self.b, steps, C.byref(ch)), "rtm_batch_autotune")
        return ch.value

    def modelling(self, nts, it_shift=-1, ntratio=1):
        nts = np.ascontiguousarray(nts, np.int32)
        if nts.size != len(self.shots):
            raise ValueError("one step count per shot")
        _lib.check(self.L.rtm_batch_modelling(self.b, nts, it_shift, ntratio), "rtm_batch_modelling")

    @property
    def last_ms(self):
        v = C.c_float()
        _lib.check(self.L.rtm_batch_last_ms(self.b, C.byref(v)), "rtm_batch_last_ms")
        return v.value


def spread_coeffs(n, x, k1, k2, nlimit, dipole=False, ntaper=0):
    """Util::CompactOrmsbySpreadCoeff + Receiver's edge taper through the C ABI;
    returns (first grid index, coefficients)."""
    L = _lib.lib()
    nl = C.c_int(nlimit)
    off = C.c_int(0)
    buf = np.zeros(max(nlimit, 1), np.float32)
    _lib.check(L.rtm_spread_coeffs(n, float(x), float(k1), float(k2), C.byref(nl), int(dipole), ntaper,
                                   buf, C.byref(off)), "rtm_spread_coeffs")
    return off.value, buf[:nl.value].copy()


class FkArgs(C.Structure):
    """rtm_fk_args (include/rtm_b200.h)."""
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nt", C.c_int), ("ntfft", C.c_int),
                ("dt", C.c_float), ("dx", C.c_float), ("dy", C.c_float), ("vsurf", C.c_float), ("z", C.c_float),
                ("trueamp", C.c_int), ("deghost", C.c_int), ("side", C.c_int), ("flcut", C.c_float),
                ("flpass", C.c_float), ("ghost_threshold", C.c_float), ("khpass", C.c_float), ("khcut", C.c_float),
                ("nlimit", C.c_int), ("domain", C.c_int), ("fmax", C.c_float)]


def fk_spread(nx, ny, nt, ntfft, dt, dx, dy, xy, traces, vsurf, z, trueamp=1, deghost=0, side=-1, flcut=0.0,
              flpass=0.0, ghost_threshold=0.1, khpass=0.4, khcut=0.48, nlimit=20, kdomain=False, fmax=60.0):
    """Receiver::spread_sdomain (or spread_kdomain) on the GPU: grid traces
    [ny][nx][nt] from traces [nr][nt] at fractional grid positions xy [nr][2]."""
    a = FkArgs(nx, ny, nt, ntfft, dt, dx, dy, vsurf, z, int(trueamp), int(deghost), int(side), flcut, flpass,
               ghost_threshold, khpass, khcut, nlimit, int(bool(kdomain)), fmax)
    xy = np.ascontiguousarray(xy, np.float32).reshape(-1, 2)
    tr = np.ascontiguousarray(traces, np.float32).reshape(len(xy), nt)
    out = np.zeros((ny, nx, nt), np.float32)
    _lib.check(_lib.lib().rtm_fk_spread(C.byref(a), len(xy), xy.ravel(), tr.ravel(), out.ravel()), "rtm_fk_spread")
    return out


class PhaseArgs(C.Structure):
    """rtm_phase_args (include/rtm_b200.h)."""
    _fields_ = [("nt", C.c_int), ("dt", C.c_float), ("Dt", C.c_float), ("t0", C.c_float), ("fmax", C.c_float),
                ("direction", C.c_int), ("w_pow", C.c_float), ("phase_deg", C.c_float), ("do_tdsp", C.c_int),
                ("nt_out", C.c_int), ("dt_out", C.c_float), ("t0_out", C.c_float), ("ntfft", C.c_int),
                ("tdsp_correction", C.c_int), ("skip_tdsp_correction", C.c_int), ("tdsp_acos_ratio", C.c_float),
                ("skip_jacobian", C.c_int), ("transform", C.c_int)]


def pad_fft_length(n):
    """The smallest even length >= n with no prime factor above 7 (stands in
    for libfftv::padfftv, which is absent from the reference tree)."""
    m = max(2, int(n) + (int(n) & 1))
    while True:
        r = m
        for p in (2, 3, 5, 7):
            while r % p == 0:
                r //= p
        if r == 1:
            return m
        m += 2


class PhaseCorrection:
    """PhaseCorrection (bgprtm/PhaseCorrection.h:11-25) on the GPU: the
    constructor's arguments, the global parameters it reads as keywords
    (tpad_ratio, tdsp_correction, skip_tdsp_correction, tdsp_acos_ratio,
    tdsp_skip_jacobian, tdsp_force_fftdft / tdsp_force_dftfft as transform 1 / 2),
    and applyForward / applyBackward on [ntr][nt] traces through
    rtm_phase_correct.  Results are returned (the reference works in place)."""
    NONE, FWD, BWD = 0, 1, 2

    def __init__(self, nt, dt, Dt, t0, fmax, direction, w_pow=0.0, phase_deg=0.0, do_tdsp=1, ntOut=-1, dtOut=-1.0,
                 t0Out=0.0, *, ntfft=None, tpad_ratio=0.5, tdsp_correction=2, skip_tdsp_correction=0,
                 tdsp_acos_ratio=0.0, skip_jacobian=False, transform=0):
        if ntfft is None:
            ntfft = pad_fft_length(int(np.rint(np.float32(nt) * np.float32(1 + tpad_ratio))))
        self.args = PhaseArgs(nt, dt, Dt, t0, fmax, direction, w_pow, phase_deg, int(do_tdsp), ntOut, dtOut, t0Out,
                              ntfft, tdsp_correction, skip_tdsp_correction, tdsp_acos_ratio, int(bool(skip_jacobian)),
                              transform)
        self.nt = nt
        self.nt_dft = ntOut if (dtOut > 0 and ntOut > 0) else nt

    def _run(self, apply, trace, ntr, nout, scaler=1.0):
        tr = np.ascontiguousarray(trace, np.float32).reshape(ntr, self.nt)
        out = np.zeros((ntr, nout), np.float32)
        _lib.check(_lib.lib().rtm_phase_correct(C.byref(self.args), apply, ntr, tr.ravel(), out.ravel(),
                                                float(scaler)), "rtm_phase_correct")
        return out

    def applyForward(self, trace, ntr):
        return self._run(1, trace, ntr, self.nt)

    def applyBackward(self, trace, ntr, scaler=1.0):
        return self._run(2, trace, ntr, self.nt_dft, scaler)


def c16_compress(a, nx, ny, nz):
    out = np.zeros((nx * nz + 2) * ny, np.uint16)
    _lib.check(_lib.lib().rtm_c16_compress(_arr(a), out, nx, ny, nz), "rtm_c16_compress")
    return out


def c16_uncompress(c, nx, ny, nz):
    out = np.zeros(nx * ny * nz, np.float32)
    _lib.check(_lib.lib().rtm_c16_uncompress(np.ascontiguousarray(c, np.uint16), out, nx, ny, nz),
               "rtm_c16_uncompress")
    return out


def w0(p: Propagator):
    return p.get(FIELD_W0)
