"""Seeded inputs of the golden fixtures (shared by tests/golden/make_golden.py
and the tests; numpy's default_rng is reproducible across platforms)."""
import numpy as np
from scipy.ndimage import gaussian_filter

from konglong_b200.spec import ENGINE_CFD, ENGINE_FD8, ENGINE_R2C, ENGINE_R2R, ISO, TTI, VTI, PropSpec

# nx*nz kept a multiple of 4: the reference's SSE loops step 4 floats across
# a y slab (bgprtm/KernelCPU.cpp:328-338).
CASES = {
    "iso_fd8": dict(engine=ENGINE_FD8, model=ISO, shape=(24, 20, 28), pml=6, steps=3, seed=11),
    "iso_fd8_nopml3d": dict(engine=ENGINE_FD8, model=ISO, shape=(24, 20, 28), pml=6, steps=3, seed=12,
                            pml3d=False),
    "vti_fd8": dict(engine=ENGINE_FD8, model=VTI, shape=(24, 20, 28), pml=6, steps=3, seed=13),
    "tti_fd8": dict(engine=ENGINE_FD8, model=TTI, shape=(24, 20, 28), pml=6, steps=3, seed=14),
    "iso_cfd": dict(engine=ENGINE_CFD, model=ISO, shape=(24, 20, 28), pml=6, steps=3, seed=15),
    "vti_cfd": dict(engine=ENGINE_CFD, model=VTI, shape=(24, 20, 28), pml=6, steps=3, seed=16),
    "tti_cfd": dict(engine=ENGINE_CFD, model=TTI, shape=(24, 20, 28), pml=6, steps=3, seed=17),
    # FFTWR2C: even lines, odd x (the isign bin n/2), odd y and z
    "iso_r2c": dict(engine=ENGINE_R2C, model=ISO, shape=(24, 20, 28), pml=6, steps=3, seed=18),
    "vti_r2c": dict(engine=ENGINE_R2C, model=VTI, shape=(23, 20, 28), pml=6, steps=3, seed=19),
    "tti_r2c": dict(engine=ENGINE_R2C, model=TTI, shape=(24, 21, 27), pml=6, steps=3, seed=20),
    # FFTWR2R: even and odd lines
    "iso_r2r": dict(engine=ENGINE_R2R, model=ISO, shape=(24, 20, 28), pml=6, steps=3, seed=21),
    "vti_r2r": dict(engine=ENGINE_R2R, model=VTI, shape=(23, 20, 28), pml=6, steps=3, seed=22),
    "tti_r2r": dict(engine=ENGINE_R2R, model=TTI, shape=(24, 21, 27), pml=6, steps=3, seed=23),
    # density models (KernelCPU::setModel's rho): ISO through the first-derivative
    # passes, the gradient divided by rho, each engine's vel * rho accumulation
    "iso_fd8_rho": dict(engine=ENGINE_FD8, model=ISO, shape=(24, 20, 28), pml=6, steps=3, seed=24, rho=True),
    "vti_fd8_rho": dict(engine=ENGINE_FD8, model=VTI, shape=(24, 20, 28), pml=6, steps=3, seed=25, rho=True),
    "tti_fd8_rho": dict(engine=ENGINE_FD8, model=TTI, shape=(24, 20, 28), pml=6, steps=3, seed=26, rho=True),
    "iso_cfd_rho": dict(engine=ENGINE_CFD, model=ISO, shape=(24, 20, 28), pml=6, steps=3, seed=27, rho=True),
    "tti_cfd_rho": dict(engine=ENGINE_CFD, model=TTI, shape=(24, 20, 28), pml=6, steps=3, seed=28, rho=True),
    "vti_r2c_rho": dict(engine=ENGINE_R2C, model=VTI, shape=(24, 20, 28), pml=6, steps=3, seed=29, rho=True),
    "iso_r2r_rho": dict(engine=ENGINE_R2R, model=ISO, shape=(24, 20, 28), pml=6, steps=3, seed=30, rho=True),
}


def case_inputs(c):
    nx, ny, nz = c["shape"]
    spec = PropSpec(nx=nx, ny=ny, nz=nz, dx=10.0, dy=10.0, dz=10.0, dt=0.001, engine=c["engine"],
                    model_type=c["model"], nbnd=(c["pml"],) * 6, vmax=4500.0, pml3d=c.get("pml3d", True))
    rng = np.random.default_rng(c["seed"])
    sh = spec.shape
    vel = (1800.0 + 2200.0 * rng.random(sh)).astype(np.float32)
    model = dict(vel=vel)
    if c["model"] >= VTI:
        model["eps"] = (0.25 * rng.random(sh)).astype(np.float32)
        model["dl"] = (0.1 * rng.random(sh)).astype(np.float32)
    if c["model"] == TTI:
        th = np.pi / 4 * rng.random(sh)
        ph = 2 * np.pi * rng.random(sh)
        model["pjx"] = (-np.sin(th) * np.cos(ph)).astype(np.float32)
        model["pjy"] = (-np.sin(th) * np.sin(ph)).astype(np.float32)
    # smooth-ish wavefields (a band-limited field like a propagating wave)
    w0 = gaussian_filter(rng.standard_normal(sh), 1.5).astype(np.float32)
    w1 = gaussian_filter(rng.standard_normal(sh), 1.5).astype(np.float32)
    if c.get("rho"):  # density 1000-2500 kg/m^3 from its own stream (the other inputs stay as they are)
        spec.use_rho = True
        model["rho"] = (1000.0 + 1500.0 * np.random.default_rng(c["seed"] + 1000).random(sh)).astype(np.float32)
    return spec, model, w0, w1


def codec_input():
    rng = np.random.default_rng(21)
    nx, ny, nz = 44, 42, 24
    a = gaussian_filter(rng.standard_normal((ny, nx, nz)), 2.0).astype(np.float32)
    a *= np.exp(-np.linspace(0, 12, ny))[:, None, None].astype(np.float32)  # decaying slabs, tiny values
    a[3] = 0.0                                 # silent slab (header zero)
    a[5, 7, 3] = np.float32(1e-30)             # below the smallest code
    a[6] *= np.float32(1e-20)                  # sub-threshold slab
    b = rng.standard_normal((8, 16, 12)).astype(np.float32)  # no tapers (small grid)
    return {"wave": (a, nx, ny, nz), "small": (b, 16, 8, 12)}


# illumination smoothing (avgVolume3D / avgVolume2D): volume shape, half widths (xy, z)
ILLUM_SMOOTH = {"grid": ((20, 24, 28), 6, 4), "line": ((1, 30, 26), 5, 7), "deep": ((12, 16, 40), 3, 10)}


def illum_input(name):
    shape = ILLUM_SMOOTH[name][0]
    rng = np.random.default_rng(100 + len(name))
    return (rng.random(shape) ** 2 * 10).astype(np.float32)


def spread_cases(count=120):
    """(n, x, k1, k2, nlimit, dipole) of the spread-kernel fixtures: Ormsby bands,
    sinc (k1 == k2) and dipole kernels, caps from 1 to 40."""
    rng = np.random.default_rng(55)
    out = []
    for _ in range(count):
        n = int(rng.integers(2, 300))
        x = float(np.float32(rng.uniform(0, n - 1)))
        k1 = float(np.float32(rng.uniform(0.05, 0.5)))
        k2 = float(np.float32(rng.uniform(k1, 0.5))) if rng.random() < 0.5 else k1
        nl = int(rng.integers(1, 40))
        dip = bool(rng.random() < 0.3) and nl >= 2
        out.append((n, x, k1, k2, nl, dip))
    return out
