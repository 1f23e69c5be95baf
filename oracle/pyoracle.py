"""ctypes bindings of the CPU checkers (TEST INFRASTRUCTURE ONLY).

`Oracle` wraps oracle/liborc.so, the C++ restatement of bgprtm's hot path
(float = the reference's FP32 order, double = the FP64 oracle).  `Reference`
wraps oracle/_ref/libbgprtm_ref.so, the reference's own CPU kernels compiled
from its sources.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg import this module; the product never does.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_SO = os.path.join(HERE, "liborc.so")
REF_SO = os.path.join(HERE, "_ref", "libbgprtm_ref.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")


def build():
    """Compile liborc.so (and oracle/_ref when the reference tree is present)."""
    import subprocess
    subprocess.run(["make", "-C", HERE, "-j8", "all"], check=True,
                   stdout=subprocess.DEVNULL)


def _load_orc():
    if not os.path.exists(ORC_SO):
        build()
    lib = C.CDLL(ORC_SO)
    vp = C.c_void_p
    lib.orc_create.restype = vp
    lib.orc_create.argtypes = [C.c_int] * 3 + [C.c_float] * 4 + [C.c_int] * 4 + [
        _i32p, C.c_float, C.c_float, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int]
    lib.orc_destroy.argtypes = [vp]
    lib.orc_set_q_coeffs.argtypes = [vp, C.c_float, _f32p, _f32p]
    optf = C.c_void_p
    lib.orc_set_model.argtypes = [vp] + [optf] * 7
    for name in ("orc_reset", "orc_kernel", "orc_update2nd", "orc_swap"):
        getattr(lib, name).argtypes = [vp]
    lib.orc_set_injection.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p,
                                      _f32p, _f32p, _f32p, _f32p, C.c_int, C.c_float]
    lib.orc_set_extraction.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p,
                                       _f32p, _f32p, _f32p, C.c_int]
    lib.orc_inject.argtypes = [vp, C.c_int]
    lib.orc_extract.argtypes = [vp, C.c_int]
    lib.orc_get_traces.argtypes = [vp, _f32p]
    lib.orc_snapshot_setup.argtypes = [vp, C.c_int, C.c_int]
    lib.orc_snapshot_store.argtypes = [vp, C.c_int]
    lib.orc_snapshot_load.argtypes = [vp, C.c_int, _f64p]
    lib.orc_image_setup.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    lib.orc_image_accumulate.argtypes = [vp, C.c_int]
    lib.orc_modelling.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    lib.orc_migration.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
    lib.orc_get.argtypes = [vp, C.c_int, _f64p]
    lib.orc_put.argtypes = [vp, C.c_int, _f32p]
    lib.orc_spread_coeffs.restype = C.c_int
    lib.orc_spread_coeffs.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float,
                                      C.POINTER(C.c_int), C.c_int, C.c_int, _f32p]
    lib.orc_c16_compress.argtypes = [_f32p, _u16p, C.c_int, C.c_int, C.c_int]
    lib.orc_c16_uncompress.argtypes = [_u16p, _f32p, C.c_int, C.c_int, C.c_int]
    lib.orc_taylor_weights.argtypes = [C.c_int, _f64p, _f64p]
    lib.orc_cfd_plan.argtypes = [C.c_int, C.c_float, C.c_int, _f32p, _f32p, _f32p]
    lib.orc_r2c_line.argtypes = [C.c_int, C.c_float, C.c_int, C.c_void_p, C.c_void_p]
    lib.orc_r2r_line.argtypes = [C.c_int, C.c_float, C.c_int, C.c_void_p, C.c_void_p]
    return lib


_orc = None


def orc_lib():
    global _orc
    if _orc is None:
        _orc = _load_orc()
    return _orc


def _ptr(a):
    return None if a is None else a.ctypes.data


class Oracle:
    """Restated bgprtm propagator on the CPU; same call sequence as the C-ABI."""

    def __init__(self, spec, double=False):
        self.lib = orc_lib()
        self.spec = spec
        s = spec
        nb = np.ascontiguousarray(s.nbnd, dtype=np.int32)
        self.h = self.lib.orc_create(s.nx, s.ny, s.nz, s.dx, s.dy, s.dz, s.dt, s.engine,
                                     s.model_type, int(s.use_q), s.q_order, nb, s.vmax,
                                     s.pml_eps, int(s.pml3d), s.pml3d_scaler, int(s.top_pml),
                                     1 if double else 0, int(getattr(s, "use_rho", False)))
        self.n = s.nx * s.ny * s.nz
        self._keep = []

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    __del__ = close

    def set_q_coeffs(self, cq0, cq, wq):
        self.lib.orc_set_q_coeffs(self.h, cq0, np.ascontiguousarray(cq, np.float32),
                                  np.ascontiguousarray(wq, np.float32))

    def set_model(self, vel, eps=None, dl=None, pjx=None, pjy=None, invq=None, rho=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32).ravel()
                for a in (vel, rho, eps, dl, pjx, pjy, invq)]
        self._keep = arrs
        self.lib.orc_set_model(self.h, *[_ptr(a) for a in arrs])

    def reset(self):
        self.lib.orc_reset(self.h)

    def kernel(self):
        self.lib.orc_kernel(self.h)

    def update2nd(self):
        self.lib.orc_update2nd(self.h)

    def swap(self):
        self.lib.orc_swap(self.h)

    def set_injection(self, ts, traces, scaler):
        self.lib.orc_set_injection(self.h, ts.ntr, ts.lx, ts.ly, ts.lz, ts.off, ts.len, ts.kx,
                                   ts.ky, ts.kz, np.ascontiguousarray(traces, np.float32),
                                   traces.shape[1], scaler)

    def set_extraction(self, ts, nt_out):
        self.nt_out, self.ntr_out = nt_out, ts.ntr
        self.lib.orc_set_extraction(self.h, ts.ntr, ts.lx, ts.ly, ts.lz, ts.off, ts.len, ts.kx,
                                    ts.ky, ts.kz, nt_out)

    def inject(self, it):
        self.lib.orc_inject(self.h, it)

    def extract(self, jt):
        self.lib.orc_extract(self.h, jt)

    def traces(self):
        out = np.zeros((self.ntr_out, self.nt_out), np.float32)
        self.lib.orc_get_traces(self.h, out)
        return out

    def snapshot_setup(self, fmt, nslots):
        self.lib.orc_snapshot_setup(self.h, fmt, nslots)

    def snapshot_store(self, slot):
        self.lib.orc_snapshot_store(self.h, slot)

    def snapshot_load(self, slot):
        out = np.zeros(self.n, np.float64)
        self.lib.orc_snapshot_load(self.h, slot, out)
        return out

    def image_setup(self, ntaper_t, ntaper_z, edge):
        self.lib.orc_image_setup(self.h, ntaper_t, ntaper_z, edge)

    def image_accumulate(self, slot):
        self.lib.orc_image_accumulate(self.h, slot)

    def modelling(self, nts, it_shift, ntratio):
        self.lib.orc_modelling(self.h, nts, it_shift, ntratio)

    def migration(self, direction, it_begin, it_end, it_shift, interval):
        self.lib.orc_migration(self.h, direction, it_begin, it_end, it_shift, interval)

    def get(self, field):
        out = np.zeros(self.n, np.float64)
        self.lib.orc_get(self.h, field, out)
        return out

    def put(self, field, a):
        self.lib.orc_put(self.h, field, np.ascontiguousarray(a, np.float32).ravel())


def spread_coeffs(n, x, k1, k2, nlimit, dipole=False, ntaper=0):
    lib = orc_lib()
    nl = C.c_int(nlimit)
    buf = np.zeros(max(nlimit, 1), np.float32)
    off = lib.orc_spread_coeffs(n, x, k1, k2, C.byref(nl), int(dipole), ntaper, buf)
    return off, buf[:nl.value].copy()


def c16_compress(a, nx, ny, nz):
    out = np.zeros((nx * nz + 2) * ny, np.uint16)
    orc_lib().orc_c16_compress(np.ascontiguousarray(a, np.float32).ravel(), out, nx, ny, nz)
    return out


def c16_uncompress(c, nx, ny, nz):
    out = np.zeros(nx * ny * nz, np.float32)
    orc_lib().orc_c16_uncompress(np.ascontiguousarray(c, np.uint16), out, nx, ny, nz)
    return out


def taylor_weights(ne):
    c1 = np.zeros(ne + 1)
    c2 = np.zeros(ne + 1)
    orc_lib().orc_taylor_weights(ne, c1, c2)
    return c1, c2


def cfd_plan(n, d, s):
    bm = np.zeros(5 * n, np.float32)
    bl = np.zeros(4 * n, np.float32)
    am = np.zeros(60, np.float32)
    orc_lib().orc_cfd_plan(n, d, s, bm, bl, am)
    return bm, bl, am


# ---------------------------------------------------------------------------
# The reference's own compiled kernels
# ---------------------------------------------------------------------------
_ref = None


def r2c_line(x, d, isign):
    """FdEngine_r2c's derivative of one line (double), the oracle's circulant."""
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros_like(x)
    orc_lib().orc_r2c_line(x.size, d, isign, x.ctypes.data, out.ctypes.data)
    return out


def r2r_line(x, d, isign):
    """FdEngine_r2r's derivative of one line (double), the oracle's matrix."""
    x = np.ascontiguousarray(x, np.float64)
    out = np.zeros_like(x)
    orc_lib().orc_r2r_line(x.size, d, isign, x.ctypes.data, out.ctypes.data)
    return out


def ref_available():
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_SO)
        vp = C.c_void_p
        lib.ref_create.restype = vp
        lib.ref_create.argtypes = [C.c_int] * 3 + [C.c_float] * 4 + [C.c_int] * 2 + [
            _i32p, C.c_float, C.c_float, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int]
        lib.ref_destroy.argtypes = [vp]
        lib.ref_set_model.argtypes = [vp] + [C.c_void_p] * 6
        for name in ("ref_reset", "ref_kernel", "ref_update2nd", "ref_swap"):
            getattr(lib, name).argtypes = [vp]
        lib.ref_put.argtypes = [vp, C.c_int, _f32p]
        lib.ref_get.argtypes = [vp, C.c_int, _f32p]
        lib.ref_set_injection.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p,
                                          _f32p, _f32p, _f32p, _f32p, C.c_int, C.c_float]
        lib.ref_inject.argtypes = [vp, C.c_int]
        lib.ref_set_extraction.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, _i32p, _i32p,
                                           _f32p, _f32p, _f32p, C.c_int]
        lib.ref_get_traces.argtypes = [vp, _f32p]
        lib.ref_modelling.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        lib.ref_run.restype = C.c_double
        lib.ref_run.argtypes = [vp, C.c_int, C.c_int]
        lib.ref_c16_compress.argtypes = [_f32p, _u16p, C.c_int, C.c_int, C.c_int]
        lib.ref_c16_uncompress.argtypes = [_u16p, _f32p, C.c_int, C.c_int, C.c_int]
        lib.ref_cfd_plan.argtypes = [C.c_int, C.c_float, C.c_int, _f32p, _f32p, _f32p]
        lib.ref_pml_coef.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                     C.c_float, _f32p]
        lib.ref_avg_volume3d.argtypes = [C.c_void_p] + [C.c_int] * 6
        lib.ref_avg_volume2d.argtypes = [C.c_void_p] + [C.c_int] * 4
        lib.ref_spread_coeffs.argtypes = [C.c_int, C.c_float, C.c_float, C.c_float, C.POINTER(C.c_int), C.c_int,
                                          _f32p]
        _ref = lib
    return _ref


class Reference:
    """The reference's KernelCPU engine (FD8 / CFD, ISO / VTI / TTI, PML)."""

    def __init__(self, spec, nthreads=0):
        self.lib = ref_lib()
        s = spec
        self.spec = s
        nb = np.ascontiguousarray(s.nbnd, dtype=np.int32)
        self.h = self.lib.ref_create(s.nx, s.ny, s.nz, s.dx, s.dy, s.dz, s.dt, s.engine,
                                     s.model_type, nb, s.vmax, s.pml_eps, int(s.pml3d),
                                     s.pml3d_scaler, int(s.top_pml), nthreads,
                                     int(getattr(s, "use_rho", False)))
        if not self.h:
            raise ValueError(f"engine {s.engine}: not a KernelCPU engine of the compiled reference")
        self.n = s.nx * s.ny * s.nz
        self._keep = []

    def close(self):
        if self.h:
            self.lib.ref_destroy(self.h)
            self.h = None

    __del__ = close

    def set_model(self, vel, eps=None, dl=None, pjx=None, pjy=None, rho=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float32).ravel()
                for a in (vel, rho, eps, dl, pjx, pjy)]
        self._keep = arrs
        self.lib.ref_set_model(self.h, *[_ptr(a) for a in arrs])

    def reset(self):
        self.lib.ref_reset(self.h)

    def kernel(self):
        self.lib.ref_kernel(self.h)

    def update2nd(self):
        self.lib.ref_update2nd(self.h)

    def swap(self):
        self.lib.ref_swap(self.h)

    def set_injection(self, ts, traces, scaler):
        self._tr = np.ascontiguousarray(traces, np.float32)
        self.lib.ref_set_injection(self.h, ts.ntr, ts.lx, ts.ly, ts.lz, ts.off, ts.len, ts.kx,
                                   ts.ky, ts.kz, self._tr, traces.shape[1], scaler)

    def inject(self, it):
        self.lib.ref_inject(self.h, it)

    def set_extraction(self, ts, nt_out):
        self._ext = (ts, nt_out)
        self.lib.ref_set_extraction(self.h, ts.ntr, ts.lx, ts.ly, ts.lz, ts.off, ts.len, ts.kx, ts.ky, ts.kz,
                                    nt_out)

    def modelling(self, nts, it_shift, ntratio):
        self.lib.ref_modelling(self.h, nts, it_shift, ntratio)

    def traces(self):
        ts, nt_out = self._ext
        out = np.zeros(ts.ntr * nt_out, np.float32)
        self.lib.ref_get_traces(self.h, out)
        return out.reshape(ts.ntr, nt_out)

    def run(self, it0, nsteps):
        return self.lib.ref_run(self.h, it0, nsteps)

    def get(self, field):
        out = np.zeros(self.n, np.float32)
        self.lib.ref_get(self.h, field, out)
        return out

    def put(self, field, a):
        self.lib.ref_put(self.h, field, np.ascontiguousarray(a, np.float32).ravel())


def ref_c16_compress(a, nx, ny, nz):
    out = np.zeros((nx * nz + 2) * ny, np.uint16)
    ref_lib().ref_c16_compress(np.ascontiguousarray(a, np.float32).ravel(), out, nx, ny, nz)
    return out


def ref_c16_uncompress(c, nx, ny, nz):
    out = np.zeros(nx * ny * nz, np.float32)
    ref_lib().ref_c16_uncompress(np.ascontiguousarray(c, np.uint16), out, nx, ny, nz)
    return out


def ref_cfd_plan(n, d, s):
    bm = np.zeros(5 * n, np.float32)
    bl = np.zeros(4 * n, np.float32)
    am = np.zeros(60, np.float32)
    ref_lib().ref_cfd_plan(n, d, s, bm, bl, am)
    return bm, bl, am


def ref_avg_volume(a, sx, sz, sy=None):
    """volumefilter.cpp's avgVolume3D (ny > 1, half widths sx, sy, sz) or
    avgVolume2D (x, z) on a copy of a [ny][nx][nz]."""
    L = ref_lib()
    v = np.ascontiguousarray(a, np.float32).copy()
    ny, nx, nz = v.shape
    if ny > 1:
        L.ref_avg_volume3d(v.ctypes.data, nx, ny, nz, sx, sx if sy is None else sy, sz)
    else:
        L.ref_avg_volume2d(v.ctypes.data, nx, nz, sx, sz)
    return v


def ref_spread_coeffs(n, x, k1, k2, nlimit, dipole=False):
    """The reference's Util::CompactOrmsbySpreadCoeff: (first index, coefficients)."""
    nl = C.c_int(nlimit)
    buf = np.zeros(max(nlimit, 1), np.float32)
    off = ref_lib().ref_spread_coeffs(n, x, k1, k2, C.byref(nl), int(dipole), buf)
    return off, buf[:nl.value].copy()


def ref_pml_coef(n, npml, d, dt, vmax, pml_eps=1e-3):
    out = np.zeros(npml, np.float32)
    ref_lib().ref_pml_coef(n, npml, d, dt, vmax, pml_eps, out)
    return out
