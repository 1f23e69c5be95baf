"""Seeded synthetic shots for the propagation path (no public data set is used).

Each builder returns a `Shot`: the PropSpec, the model volumes in the
reference layout ([ny][nx][nz], z fastest), the source wavelet and the
source / receiver spread kernels.  `scale` shrinks the grid for tests while
keeping the structure.  Sizes, spacings, frequencies and value ranges follow
the five workloads the project is measured on:
  iso128   : 128^3 ISO, FD8, 1000 steps, PML 20, 4 layers + 5 % smooth noise
  vti_cfd  : 512x512x400 VTI, compact FD, 4000 steps, PML 32, 256x256 receivers
  tti_q    : 640x640x512 TTI + Q, 5000 steps, PML 32 (assumed)
  batch    : 64 small ISO/VTI shots of uneven aperture (96-256 cells per axis)
CFL: the time step is min(stated dt, the stability rule of
ModelPrepare::calcDeltaTime, bgprtm/ModelPrepare.cpp:647-914), as the
reference itself only accepts a user dt below its stability bound
(bgprtm/ModelPrepare.cpp:901-910).
"""
from dataclasses import dataclass, field

import numpy as np

from .spec import (ENGINE_CFD, ENGINE_CFDB, ENGINE_FD8, ENGINE_FFTV, ENGINE_R2C, ENGINE_R2R, ENGINE_SINCOS, ISO, TTI,
                   VTI, PropSpec, TraceSet)


@dataclass
class Shot:
    spec: PropSpec
    nt: int                      # recorded time samples (steps)
    vel: np.ndarray
    eps: np.ndarray = None
    dl: np.ndarray = None
    pjx: np.ndarray = None
    pjy: np.ndarray = None
    invq: np.ndarray = None
    wavelet: np.ndarray = None   # [nt]
    src_pos: tuple = None        # fractional grid index (x, y, z)
    rcv_pos: np.ndarray = None   # [nr, 3]
    interval: int = 4            # snapshot interval (steps)
    fpeak: float = 15.0
    name: str = ""
    extra: dict = field(default_factory=dict)

    def model_arrays(self):
        return dict(vel=self.vel, eps=self.eps, dl=self.dl, pjx=self.pjx, pjy=self.pjy, invq=self.invq)


# ---------------------------------------------------------------------------
def smooth_field(shape, sigma, rng):
    """N(0,1) noise Gaussian-smoothed with `sigma` cells, scaled to max|g| = 1."""
    from scipy.ndimage import gaussian_filter, zoom
    n = int(np.prod(shape))
    if n <= 8_000_000 or sigma < 4:
        g = gaussian_filter(rng.standard_normal(shape).astype(np.float32), sigma, mode="reflect")
    else:
        f = 4
        small = tuple(max(4, s // f) for s in shape)
        g = gaussian_filter(rng.standard_normal(small).astype(np.float32), sigma / f, mode="reflect")
        g = zoom(g, [s / c for s, c in zip(shape, small)], order=1)[:shape[0], :shape[1], :shape[2]]
        g = np.ascontiguousarray(g, dtype=np.float32)
    m = np.abs(g).max()
    return (g / m if m > 0 else g).astype(np.float32)


def minmax(g, lo, hi):
    a, b = float(g.min()), float(g.max())
    return (lo + (g - a) * ((hi - lo) / (b - a if b > a else 1.0))).astype(np.float32)


def ricker(f, dt, nt, delay=None):
    """Ricker wavelet, peak frequency f, delayed by 1/f, amplitude x 1e5 as
    Wavelet.cpp scales its wavelets (bgprtm/Wavelet.cpp:74-78)."""
    t0 = 1.0 / f if delay is None else delay
    t = np.arange(nt) * dt - t0
    a = (np.pi * f * t) ** 2
    return ((1.0 - 2.0 * a) * np.exp(-a) * 1e5).astype(np.float32)


def fd8_k1max():
    """FdEngine_fd::get_k1max with Taylor weights (bgprtm/FdEngine_fd.cpp:69-81)."""
    c2 = [-205 / 72, 8 / 5, -1 / 5, 8 / 315, -1 / 560]
    s = -c2[0]
    sg = 2
    for j in range(1, 5):
        s += sg * c2[j]
        sg = -sg
    return float(np.sqrt(np.float32(s)) * np.float32(1.01))


def cfl_dt(spec: PropSpec, vel, eps=None, dl=None, pjx=None, pjy=None, invq=None, maxfreq=None, rho=None,
           qref=None):
    """ModelPrepare::calcDeltaTime restated (bgprtm/ModelPrepare.cpp:647-881)
    for a rectangular grid.  k1max: FdEngine_fd::get_k1max for the FD engine
    (bgprtm/FdEngine_fd.cpp:69-81), pi otherwise (:652-654).  Per cell:
      ISO  lambda = v sqrt(rdx2 + rdy2 + rdz2)                        (:702-716)
      VTI  tmp = (1 + 2e)(rdx2 + rdy2) + rdz2,
           lambda = v sqrt((tmp + sqrt(tmp^2 - 8 (e - d)(rdx2 + rdy2) rdz2)) / 2),
           dt_cell = 2 / k1max / lambda / sqrt(1 + 2e)                (:741-757)
      TTI  the wavenumbers 1/dx, 1/dy, 1/dz rotated into the symmetry axis
           frame (sin theta = |(pjx, pjy)|, cos phi = -pjx / sin theta,
           sin phi = -pjy / sin theta), then the largest VTI lambda over the
           axis combinations ic = 1 .. nc-1 (nc 8 in 3-D, 4 in 2-D)   (:838-881)
    With a density model lambda is multiplied by sqrt(rho) per cell and the
    minimum dt by sqrt(min rho) (:679-700, :720-738, :795-836).  With Q:
    dt *= 1 - max(1/Q) (3 + 2/pi ln(maxfreq / qref)), qref = maxfreq / 3 by
    default (:885-891)."""
    k1 = fd8_k1max() if spec.engine == ENGINE_FD8 else float(np.float32(np.pi))
    three_d = spec.ny > 1
    v = np.asarray(vel, np.float64).ravel()
    sr = np.sqrt(np.asarray(rho, np.float64).ravel()) if rho is not None else 1.0
    rdx2, rdz2 = 1.0 / spec.dx ** 2, 1.0 / spec.dz ** 2
    rdy2 = 1.0 / spec.dy ** 2 if three_d else 0.0
    if spec.model_type == ISO or eps is None:
        lam = v * sr * np.sqrt(rdx2 + rdy2 + rdz2)
        dt = float(np.min(2.0 / k1 / lam))
    else:
        e = np.asarray(eps, np.float64).ravel()
        d = np.asarray(dl, np.float64).ravel()
        if spec.model_type == VTI or pjx is None:
            h2 = rdx2 + rdy2
            tmp = (1 + 2 * e) * h2 + rdz2
            lam = v * np.sqrt((tmp + np.sqrt(np.maximum(tmp * tmp - 8 * (e - d) * h2 * rdz2, 0))) / 2)
        else:
            px_ = np.asarray(pjx, np.float64).ravel()
            py_ = np.asarray(pjy, np.float64).ravel() if pjy is not None else np.zeros_like(px_)
            st = np.sqrt(px_ * px_ + py_ * py_)
            ct = np.sqrt(np.maximum(1 - st * st, 0))
            big = st > 1e-15
            cp = np.where(big, -px_ / np.where(big, st, 1), 1.0)
            sp = np.where(big, -py_ / np.where(big, st, 1), 0.0)
            akx, aky, akz = 1 / spec.dx, 1 / spec.dy, 1 / spec.dz
            rx = (cp * ct * akx + sp * ct * aky - st * akz) ** 2
            ry = (-sp * akx + cp * aky) ** 2 if three_d else np.zeros_like(v)
            rz = (cp * st * akx + sp * st * aky + ct * akz) ** 2
            lam = np.zeros_like(v)
            for ic in range(1, 8 if three_d else 4):
                icz, icx, icy = ic & 1, (ic >> 1) & 1, (ic >> 2) & 1
                h2 = rx * icx + ry * icy
                z2 = rz * icz
                t1 = (1 + 2 * e) * h2 + z2
                lam = np.maximum(lam, v * np.sqrt((t1 + np.sqrt(np.maximum(t1 * t1 - 8 * (e - d) * h2 * z2, 0))) / 2))
        lam = lam * sr
        dt = float(np.min(2.0 / k1 / lam / np.sqrt(1 + 2 * e)))
    if rho is not None:
        dt *= float(np.sqrt(np.min(np.asarray(rho, np.float64))))
    if spec.use_q and invq is not None and maxfreq:
        qr = maxfreq / 3 if qref is None else qref
        dt *= 1 - float(np.max(invq)) * (3 + 2 / np.pi * np.log(maxfreq / qr))
    return dt


def update_zlimit(iz_min, iz_max, nz, spread):
    """Receiver::update_zrange's limit on the z spread (bgprtm/Receiver.cpp:129-161)."""
    lim = min(iz_min + 1, nz - 1 - iz_max)
    if lim < spread:
        spread = max(5, lim)
    iz0 = iz_min - spread + 1
    iz1 = iz_max + spread
    return iz1 - iz0 + 1


def make_traceset(points, nx, ny, nz, spread, k1, k2, coeff_fn, ntaper_xy=10):
    """Receiver::spreadCoeffs (bgprtm/Receiver.cpp:306-363): separable kernels
    per point.  points: [n, 3] fractional grid indices (x, y, z)."""
    pts = np.asarray(points, np.float64).reshape(-1, 3)
    n = len(pts)
    izs = np.floor(pts[:, 2]).astype(int)
    lz_cap = update_zlimit(int(izs.min()), int(izs.max()), nz, spread)
    lx_cap = 1 if nx == 1 else max(1, 2 * spread)
    ly_cap = 1 if ny == 1 else max(1, 2 * spread)
    off = np.zeros((n, 3), np.int32)
    ln = np.zeros((n, 3), np.int32)
    kx = np.zeros((n, lx_cap), np.float32)
    ky = np.zeros((n, ly_cap), np.float32)
    kz = np.zeros((n, lz_cap), np.float32)
    for r, (x, y, z) in enumerate(pts):
        o, c = coeff_fn(nx, np.float32(x), k1, k2, lx_cap, False, ntaper_xy)
        off[r, 0], ln[r, 0], kx[r, :len(c)] = o, len(c), c
        o, c = coeff_fn(ny, np.float32(y), k1, k2, ly_cap, False, ntaper_xy)
        off[r, 1], ln[r, 1], ky[r, :len(c)] = o, len(c), c
        o, c = coeff_fn(nz, np.float32(z), k1, k2, lz_cap, False, 0)
        off[r, 2], ln[r, 2], kz[r, :len(c)] = o, len(c), c
    return TraceSet(n, lx_cap, ly_cap, lz_cap, off, ln, kx, ky, kz)


def spread_band(spec: PropSpec):
    """src_apply_khpass / khcut defaults (bgprtm/ModelRegrid.cpp:86-87) from the
    engine's dispersion factor (bgprtm/FdEngine.cpp:241-256)."""
    if spec.engine in (ENGINE_CFD, ENGINE_CFDB):  # names starting with "CFD" take the compact-FD factor
        disp = 0.9
    elif spec.engine in (ENGINE_R2C, ENGINE_R2R, ENGINE_FFTV, ENGINE_SINCOS):
        disp = 1.0  # pseudo-spectral engines keep FdEngine::getFdDispersion's default
    else:
        disp = 0.46 if spec.model_type >= VTI else 0.6
    k = disp * 0.5 if disp <= 0.8 else None
    return (k, k) if k is not None else (0.40, 0.48)


# ---------------------------------------------------------------------------
def iso128(scale=1.0, seed=1, nt=1000):
    rng = np.random.default_rng(seed)
    n = max(32, int(round(128 * scale)))
    pml = max(6, int(round(20 * scale)))
    spec = PropSpec(nx=n, ny=n, nz=n, dx=10.0, dy=10.0, dz=10.0, dt=0.001, engine=ENGINE_FD8, model_type=ISO,
                    nbnd=(pml,) * 6, vmax=4500.0)
    iz = np.arange(n)
    layer_v = np.array([1500, 2200, 3000, 4500], np.float32)
    prof = layer_v[np.minimum(iz * 4 // n, 3)]
    vel = np.broadcast_to(prof, spec.shape).astype(np.float32)
    g = smooth_field(spec.shape, 5.0, rng)
    # 5 % perturbation, clipped to the layer range so dt = 1 ms meets the FD8 CFL bound
    vel = np.clip(vel * (1.0 + 0.05 * g), 1500.0, 4500.0).astype(np.float32)
    # dt = 1 ms as stated: v dt / dx = 0.45 is inside the FD8 leapfrog bound 0.4529
    # (the reference's rule adds a 1 % margin on k1max, which would give 0.996 ms)
    src = (n / 2, n / 2, pml + 1)
    nr = max(4, int(round(64 * scale)))
    step = max(1, (n - 2) // nr)
    rx = 1 + step * np.arange(nr)
    rxx, ryy = np.meshgrid(rx, rx, indexing="xy")
    rcv = np.stack([rxx.ravel(), ryy.ravel(), np.full(rxx.size, pml + 2.0)], 1).astype(np.float32)
    return Shot(spec, nt, vel, wavelet=ricker(15.0, spec.dt, nt), src_pos=src, rcv_pos=rcv, interval=4,
                fpeak=15.0, name="iso128")


def small_shots(nshots=64, seed=4, size=(96, 256), steps=(500, 2000), nrec=16, model=ISO):
    """Batched small-shot workload: every shot draws its grid (each axis
    uniform in `size`), step count, 3-5 flat layers between 1500 and 4500 m/s
    and a 10-25 Hz Ricker source from one seed.  10 m spacing, dt = 1 ms (inside
    the FD8 leapfrog bound at 4500 m/s), PML 16, source at the surface centre,
    nrec x nrec receivers two cells below the top PML.  model=VTI adds a
    Thomsen epsilon in [0, 0.2] and delta in [0, 0.1] per layer, and each shot
    takes the time step of the CFL rule (at most 1 ms), since epsilon raises
    the horizontal velocity."""
    rng = np.random.default_rng(seed)
    shots = []
    for k in range(nshots):
        nx, ny, nz = (int(v) for v in rng.integers(size[0], size[1] + 1, 3))
        nt = int(rng.integers(steps[0], steps[1] + 1))
        pml = 16
        spec = PropSpec(nx=nx, ny=ny, nz=nz, dx=10.0, dy=10.0, dz=10.0, dt=0.001, engine=ENGINE_FD8, model_type=model,
                        nbnd=(pml,) * 6, vmax=4500.0)
        nl = int(rng.integers(3, 6))
        vals = np.sort(rng.uniform(1500.0, 4500.0, nl)).astype(np.float32)
        cuts = np.sort(rng.uniform(0.1, 0.9, nl - 1)) * nz
        layer = np.searchsorted(cuts, np.arange(nz))
        vel = np.ascontiguousarray(np.broadcast_to(vals[layer], spec.shape), np.float32)
        eps = dl = None
        if model == VTI:
            ev = rng.uniform(0.0, 0.2, nl).astype(np.float32)
            dv = np.minimum(rng.uniform(0.0, 0.1, nl), ev).astype(np.float32)
            eps = np.ascontiguousarray(np.broadcast_to(ev[layer], spec.shape), np.float32)
            dl = np.ascontiguousarray(np.broadcast_to(dv[layer], spec.shape), np.float32)
            spec.dt = float(min(0.001, cfl_dt(spec, vel, eps, dl)))
        f = float(rng.uniform(10.0, 25.0))
        step_x, step_y = max(1, (nx - 2) // nrec), max(1, (ny - 2) // nrec)
        rxx, ryy = np.meshgrid(1 + step_x * np.arange(nrec), 1 + step_y * np.arange(nrec), indexing="xy")
        rcv = np.stack([rxx.ravel(), ryy.ravel(), np.full(rxx.size, pml + 2.0)], 1).astype(np.float32)
        shots.append(Shot(spec, nt, vel, eps=eps, dl=dl, wavelet=ricker(f, spec.dt, nt), src_pos=(nx / 2, ny / 2, pml + 1),
                          rcv_pos=rcv, interval=4, fpeak=f, name=f"small{k}"))
    return shots


def vti_cfd(scale=1.0, seed=2, nt=4000):
    rng = np.random.default_rng(seed)
    nx = max(32, int(round(512 * scale)))
    nz = max(32, int(round(400 * scale)))
    pml = max(6, int(round(32 * scale)))
    spec = PropSpec(nx=nx, ny=nx, nz=nz, dx=10.0, dy=10.0, dz=10.0, dt=0.0008, engine=ENGINE_CFD,
                    model_type=VTI, nbnd=(pml,) * 6, vmax=4500.0)
    # smooth layered velocity: 6 seeded interfaces, 1500 -> 4500 m/s, smoothed
    cuts = np.sort(rng.uniform(0.1, 0.9, 5)) * nz
    vals = np.linspace(1500, 4500, 6).astype(np.float32)
    iz = np.arange(nz)
    prof = vals[np.searchsorted(cuts, iz)]
    from scipy.ndimage import gaussian_filter1d
    prof = gaussian_filter1d(prof.astype(np.float32), 3.0)
    lat = smooth_field(spec.shape, 8.0, rng)
    vel = np.clip(prof[None, None, :] * (1.0 + 0.03 * lat), 1500.0, 4500.0).astype(np.float32)
    eps = minmax(smooth_field(spec.shape, 8.0, rng), 0.0, 0.25)
    dl = minmax(smooth_field(spec.shape, 8.0, rng), 0.0, 0.10)
    spec.dt = float(min(spec.dt, cfl_dt(spec, vel, eps, dl)))
    src = (nx / 2, nx / 2, pml + 1)
    nr = max(4, int(round(256 * scale)))
    step = max(1, (nx - 2) // nr)
    rx = 1 + step * np.arange(nr)
    rxx, ryy = np.meshgrid(rx, rx, indexing="xy")
    rcv = np.stack([rxx.ravel(), ryy.ravel(), np.full(rxx.size, pml + 2.0)], 1).astype(np.float32)
    return Shot(spec, nt, vel, eps=eps, dl=dl, wavelet=ricker(20.0, spec.dt, nt), src_pos=src, rcv_pos=rcv,
                interval=8, fpeak=20.0, name="vti_cfd")


def tti_q(scale=1.0, seed=3, nt=5000, engine=ENGINE_FD8):
    rng = np.random.default_rng(seed)
    nx = max(32, int(round(640 * scale)))
    nz = max(32, int(round(512 * scale)))
    pml = max(6, int(round(32 * scale)))
    spec = PropSpec(nx=nx, ny=nx, nz=nz, dx=10.0, dy=10.0, dz=10.0, dt=0.001, engine=engine, model_type=TTI,
                    use_q=True, q_order=4, nbnd=(pml,) * 6, vmax=4500.0)
    iz = np.arange(nz)
    prof = (1500.0 + 3000.0 * iz / max(1, nz - 1)).astype(np.float32)
    lat = smooth_field(spec.shape, 8.0, rng)
    vel = np.clip(prof[None, None, :] * (1.0 + 0.03 * lat), 1500.0, 4500.0).astype(np.float32)
    eps = minmax(smooth_field(spec.shape, 8.0, rng), 0.0, 0.25)
    dl = minmax(smooth_field(spec.shape, 8.0, rng), 0.0, 0.10)
    theta = np.deg2rad(minmax(smooth_field(spec.shape, 8.0, rng), 0.0, 45.0))
    phi = np.deg2rad(minmax(smooth_field(spec.shape, 8.0, rng), 0.0, 360.0))
    pjx = (-np.sin(theta) * np.cos(phi)).astype(np.float32)   # bgprtm/ModelLoader.cpp:303-325
    pjy = (-np.sin(theta) * np.sin(phi)).astype(np.float32)
    q = minmax(smooth_field(spec.shape, 8.0, rng), 30.0, 200.0)
    invq = (1.0 / q).astype(np.float32)
    spec.dt = float(min(spec.dt, cfl_dt(spec, vel, eps, dl, pjx, pjy, invq, maxfreq=60.0)))
    src = (nx / 2, nx / 2, pml + 1)
    nr = max(4, int(round(128 * scale)))
    step = max(1, (nx - 2) // nr)
    rx = 1 + step * np.arange(nr)
    rxx, ryy = np.meshgrid(rx, rx, indexing="xy")
    rcv = np.stack([rxx.ravel(), ryy.ravel(), np.full(rxx.size, pml + 2.0)], 1).astype(np.float32)
    return Shot(spec, nt, vel, eps=eps, dl=dl, pjx=pjx, pjy=pjy, invq=invq,
                wavelet=ricker(20.0, spec.dt, nt), src_pos=src, rcv_pos=rcv, interval=8, fpeak=20.0,
                name="tti_q")


# Order-4 seed of Q::fitQCoeff for q_amp == 1 (bgprtm/Q.cpp:176-177) pushed
# through the wave-equation transform of bgprtm/Q.cpp:275-290 (the levmar fit
# itself is bypassed: fixed coefficients).
Q_SEED4 = [2.0832741, -0.040106162, -0.21464862, -1.0239593, -9.7581205, 0.024538578, 0.18895587,
           1.0043846, 6.2038145]


def q_coefficients(dt, fdom, order=4):
    c = np.array(Q_SEED4, np.float32)
    w0_dt = np.float32(2 * np.pi) * np.float32(fdom) * np.float32(dt)
    # the seed is taken as the fitted result (absolute w_l, as after postFitAdjust)
    cq = c[1:order + 1].copy()
    wq = c[order + 1:2 * order + 1].copy()
    for i in range(order):
        wn = wq[i] * w0_dt
        cq[i] = cq[i] * np.float32(np.exp(-wn)) * 2 * w0_dt
        wq[i] = np.float32(np.exp(-2 * wn))
    return float(c[0]), cq.astype(np.float32), wq.astype(np.float32)
