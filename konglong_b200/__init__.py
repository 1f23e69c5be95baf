"""B200-native reverse-time-migration propagation and imaging engine.

The hot path of UPC-HPC/konglong's bgprtm (KernelCPU / FdEngine_fd /
FdEngine_cfd / PML / Receiver / WaveFieldCompress / ImagingCorrelator) as
hand-written sm_100a CUDA kernels behind the C ABI of include/rtm_b200.h.
"""
from .spec import (BACKWARD, ENGINE_CFD, ENGINE_CFDB, ENGINE_FD8, ENGINE_FFTV, ENGINE_R2C, ENGINE_R2R, ENGINE_SINCOS, FIELD_IMAGE, FIELD_INVQ, FIELD_VEL, FIELD_W0,
                   FIELD_W1, FORWARD, ISO, SNAP_C16, SNAP_FP16S, SNAP_FP32, TTI, VTI, PropSpec, TraceSet)

__all__ = ["PropSpec", "TraceSet", "Propagator", "ENGINE_FD8", "ENGINE_CFD", "ENGINE_R2C", "ENGINE_R2R", "ENGINE_CFDB",
           "ENGINE_FFTV", "ENGINE_SINCOS", "ISO", "VTI", "TTI",
           "FORWARD", "BACKWARD", "SNAP_FP32", "SNAP_C16", "SNAP_FP16S", "FIELD_W0", "FIELD_W1",
           "FIELD_VEL", "FIELD_IMAGE", "FIELD_INVQ"]


def __getattr__(name):
    if name in ("Propagator", "spread_coeffs", "c16_compress", "c16_uncompress"):
        from . import propagator
        return getattr(propagator, name)
    raise AttributeError(name)
