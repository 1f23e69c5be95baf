"""Propagation set-up shared by the host driver, the tests and the bench.

`PropSpec` carries what bgprtm's KernelCPU/FdEngine constructor and
setBoundary take (bgprtm/KernelCPU.h:19-27, bgprtm/FdEngine.cpp:24-53,
108-182) and maps one-to-one onto the C ABI's rtm_dims + rtm_config.
`TraceSet` is the packed form of Receiver::spreadCoeffs' per-trace separable
kernels (kernels_x/y/z, offxs/offys/offzs, lxs/lys/lzs,
bgprtm/Receiver.h:154-156).
"""
from dataclasses import dataclass, field

import numpy as np

# FD::FD, CFD, FFTWR2C, FFTWR2R, CFD_BATCH, FFTV, SINCOS
ENGINE_FD8, ENGINE_CFD, ENGINE_R2C, ENGINE_R2R, ENGINE_CFDB, ENGINE_FFTV, ENGINE_SINCOS = 0, 1, 2, 3, 4, 5, 6
ISO, VTI, TTI = 1, 2, 3
FORWARD, BACKWARD = 0, 1
SNAP_FP32, SNAP_C16, SNAP_FP16S, SNAP_AE = 0, 1, 2, 3
FIELD_W0, FIELD_W1, FIELD_VEL, FIELD_IMAGE, FIELD_INVQ, FIELD_ILLUM = 0, 1, 2, 3, 4, 5
IC_IMAGE1, IC_INVERSION = 0, 1


@dataclass
class PropSpec:
    nx: int
    ny: int
    nz: int
    dx: float = 10.0
    dy: float = 10.0
    dz: float = 10.0
    dt: float = 0.001
    engine: int = ENGINE_FD8
    model_type: int = ISO
    use_q: bool = False
    q_order: int = 4
    nbnd: tuple = (20, 20, 20, 20, 20, 20)   # x1, x2, y1, y2, z1, z2
    vmax: float = 4500.0
    pml_eps: float = 1e-3
    pml3d: bool = True
    pml3d_scaler: float = 0.3
    top_pml: bool = True
    state_fp16: bool = False
    use_rho: bool = False         # density model (KernelCPU::setModel's rho)
    q_bf16: bool = False          # Q memory variables stored as bfloat16
    kernel_variant: int = 0       # 0 auto, 1 one cell per thread / plain tiles, 2 TMA (CFD x/y tiles,
                                  # ISO one-cell plane pipeline), 3 FD8 4 z cells per thread with TMA
                                  # rings, 4 ISO 4 z cells with register prefetch, 5 compact FD with
                                  # streamed x / y lines, 6 / 8 compact FD segment-parallel with
                                  # plain / TMA tile loads, 7 as 3 with the Q update loading its own
                                  # operands, 9 compact FD with the z line solves carrying the epilogues'
                                  # interior cells

    @property
    def n(self):
        return self.nx * self.ny * self.nz

    @property
    def shape(self):
        """numpy shape of a volume in the reference layout (z fastest)."""
        return (self.ny, self.nx, self.nz)

    @property
    def dt_dxyz(self):
        """Receiver::dt_dxyz for a 3-D grid (bgprtm/Receiver.cpp:55-57)."""
        return np.float32(1.0) / np.float32(self.dz) / np.float32(self.dx) / np.float32(self.dy)


@dataclass
class TraceSet:
    """Separable spread kernels of ntr traces, padded to fixed strides."""
    ntr: int
    lx: int
    ly: int
    lz: int
    off: np.ndarray = field(repr=False)   # int32 [ntr, 3] first index x, y, z
    len: np.ndarray = field(repr=False)   # int32 [ntr, 3] used length x, y, z
    kx: np.ndarray = field(repr=False)    # float32 [ntr, lx]
    ky: np.ndarray = field(repr=False)    # float32 [ntr, ly]
    kz: np.ndarray = field(repr=False)    # float32 [ntr, lz]
