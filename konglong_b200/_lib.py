"""ctypes binding of the in-tree CUDA library konglong_b200/_rtm_b200.so.

The C ABI is declared in include/rtm_b200.h.  There is no CPU fallback: if the
library is missing or fails to load, import-time use raises RuntimeError.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_rtm_b200.so")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")

RTM_OK = 0
STATUS = {0: "RTM_OK", -1: "RTM_ERR_ARG", -2: "RTM_ERR_STATE", -3: "RTM_ERR_CUDA",
          -4: "RTM_ERR_NOMEM", -5: "RTM_ERR_UNSUPPORTED", -6: "RTM_ERR_NONFINITE",
          -7: "RTM_ERR_TIMEOUT"}
STATUS_CODE = {v: k for k, v in STATUS.items()}

# every entry point of include/rtm_b200.h
EXPORTS = ["rtm_config_default", "rtm_create", "rtm_destroy", "rtm_last_error", "rtm_set_q_coeffs",
           "rtm_set_model", "rtm_reset", "rtm_kernel", "rtm_update2nd", "rtm_swap",
           "rtm_spread_coeffs", "rtm_r2r_line_matrix", "rtm_fk_spread", "rtm_phase_correct", "rtm_set_injection", "rtm_set_extraction", "rtm_inject",
           "rtm_extract", "rtm_get_traces", "rtm_snapshot_setup", "rtm_snapshot_store",
           "rtm_snapshot_load", "rtm_image_setup", "rtm_image_accumulate", "rtm_modelling",
           "rtm_migration", "rtm_get", "rtm_put", "rtm_c16_compress", "rtm_c16_uncompress",
           "rtm_last_loop_ms", "rtm_last_loop_launches", "rtm_profile", "rtm_profile_read",
           "rtm_c16_compress_noalloc", "rtm_autotune", "rtm_autotune_result", "rtm_snapshot_offload", "rtm_illum_setup", "rtm_image_condition", "rtm_image_double", "rtm_get_image_double", "rtm_get_illum_double", "rtm_set_compressor_fallback", "rtm_illum_compensate", "rtm_check_finite", "rtm_selftest_bounded_wait",
           "rtm_batch_create", "rtm_batch_destroy", "rtm_batch_modelling", "rtm_batch_last_ms",
           "rtm_batch_autotune", "rtm_ae_nparams", "rtm_ae_create", "rtm_ae_destroy", "rtm_ae_set_params",
           "rtm_ae_get_params", "rtm_ae_loss_grad", "rtm_ae_train_step", "rtm_ae_reconstruct",
           "rtm_ae_compress_volume", "rtm_ae_decompress_volume", "rtm_set_compressor",
           "rtm_snapshot_window", "rtm_snapshot_slot_bytes", "rtm_checkpoint_setup", "rtm_checkpoint_save", "rtm_checkpoint_load"]

KERNEL_KINDS = ["iso_fd8_step", "grad_fd8", "div_fd8", "cfd_z", "cfd_x", "cfd_y", "cfd_grad_epilogue",
                "cfd_div_epilogue", "inject", "extract", "slab_max", "fused_io", "cfd_y_fused", "cfd_x_fused"]


class RtmDims(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_float),
                ("dy", C.c_float), ("dz", C.c_float), ("dt", C.c_float)]


class RtmConfig(C.Structure):
    _fields_ = [("engine", C.c_int), ("model_type", C.c_int), ("use_q", C.c_int),
                ("q_order", C.c_int), ("nbnd", C.c_int * 6), ("vmax", C.c_float),
                ("pml_eps", C.c_float), ("pml3d", C.c_int), ("pml3d_scaler", C.c_float),
                ("top_pml", C.c_int), ("state_fp16", C.c_int), ("kernel_variant", C.c_int),
                ("use_rho", C.c_int), ("q_bf16", C.c_int)]


class RtmError(RuntimeError):
    def __init__(self, code, what, detail=""):
        self.code = code
        super().__init__(f"{what} failed: {STATUS.get(code, code)}" + (f" ({detail})" if detail else ""))


_lib = None


def lib():
    """Load the CUDA library (built by konglong_b200.build / __graft_entry__.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m konglong_b200.build` "
                           "(the CUDA path has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    i = C.c_int
    f = C.c_float
    L.rtm_config_default.argtypes = [C.POINTER(RtmConfig)]
    L.rtm_config_default.restype = None
    L.rtm_create.argtypes = [C.POINTER(RtmDims), C.POINTER(RtmConfig), C.POINTER(vp)]
    L.rtm_destroy.argtypes = [vp]
    L.rtm_last_error.argtypes = [vp]
    L.rtm_last_error.restype = C.c_char_p
    L.rtm_set_q_coeffs.argtypes = [vp, f, _f32p, _f32p]
    L.rtm_set_model.argtypes = [vp] + [vp] * 7
    for name in ("rtm_reset", "rtm_kernel", "rtm_update2nd", "rtm_swap"):
        getattr(L, name).argtypes = [vp]
    L.rtm_spread_coeffs.argtypes = [i, f, f, f, C.POINTER(i), i, i, _f32p, C.POINTER(i)]
    L.rtm_r2r_line_matrix.argtypes = [i, f, i, _f32p]
    L.rtm_fk_spread.argtypes = [vp, i, _f32p, _f32p, _f32p]
    L.rtm_phase_correct.argtypes = [vp, i, i, _f32p, _f32p, f]
    L.rtm_set_injection.argtypes = [vp, i, i, i, i, _i32p, _i32p, _f32p, _f32p, _f32p, _f32p, i, f]
    L.rtm_set_extraction.argtypes = [vp, i, i, i, i, _i32p, _i32p, _f32p, _f32p, _f32p, i]
    L.rtm_inject.argtypes = [vp, i]
    L.rtm_extract.argtypes = [vp, i]
    L.rtm_get_traces.argtypes = [vp, _f32p]
    L.rtm_snapshot_setup.argtypes = [vp, i, i]
    L.rtm_snapshot_store.argtypes = [vp, i]
    L.rtm_snapshot_load.argtypes = [vp, i, _f32p]
    L.rtm_image_setup.argtypes = [vp, i, i, i]
    L.rtm_image_accumulate.argtypes = [vp, i]
    L.rtm_modelling.argtypes = [vp, i, i, i]
    L.rtm_migration.argtypes = [vp, i, i, i, i, i]
    L.rtm_get.argtypes = [vp, i, vp]
    L.rtm_put.argtypes = [vp, i, vp]
    L.rtm_c16_compress.argtypes = [_f32p, _u16p, i, i, i]
    L.rtm_c16_uncompress.argtypes = [_u16p, _f32p, i, i, i]
    L.rtm_last_loop_ms.argtypes = [vp, C.POINTER(f)]
    L.rtm_c16_compress_noalloc.argtypes = [vp, vp, i, i, i, vp]
    L.rtm_autotune.argtypes = [vp, i, C.POINTER(i)]
    L.rtm_autotune_result.argtypes = [vp, i, C.POINTER(i), C.POINTER(C.c_float)]
    L.rtm_snapshot_offload.argtypes = [vp, i]
    L.rtm_snapshot_window.argtypes = [vp, i]
    L.rtm_snapshot_slot_bytes.argtypes = [vp, i, C.POINTER(C.c_size_t)]
    L.rtm_checkpoint_setup.argtypes = [vp, i, C.POINTER(C.c_size_t)]
    L.rtm_checkpoint_save.argtypes = [vp, i]
    L.rtm_checkpoint_load.argtypes = [vp, i]
    L.rtm_illum_setup.argtypes = [vp, i]
    L.rtm_image_condition.argtypes = [vp, i]
    L.rtm_image_double.argtypes = [vp, i, i, i, f, f]
    L.rtm_get_image_double.argtypes = [vp, vp]
    L.rtm_get_illum_double.argtypes = [vp, vp]
    L.rtm_set_compressor_fallback.argtypes = [vp, C.c_float, C.c_float]
    L.rtm_illum_compensate.argtypes = [vp, i, i, C.c_float, C.c_float]
    L.rtm_check_finite.argtypes = [vp, i, C.POINTER(i)]
    L.rtm_selftest_bounded_wait.argtypes = [vp]
    L.rtm_batch_create.argtypes = [C.POINTER(vp), i, C.POINTER(vp)]
    L.rtm_batch_destroy.argtypes = [vp]
    L.rtm_batch_modelling.argtypes = [vp, _i32p, i, i]
    L.rtm_batch_last_ms.argtypes = [vp, C.POINTER(f)]
    L.rtm_batch_autotune.argtypes = [vp, i, C.POINTER(i)]
    L.rtm_ae_nparams.argtypes = []
    L.rtm_ae_create.argtypes = [C.POINTER(vp)]
    L.rtm_ae_destroy.argtypes = [vp]
    L.rtm_ae_set_params.argtypes = [vp, _f32p]
    L.rtm_ae_get_params.argtypes = [vp, _f32p]
    L.rtm_ae_loss_grad.argtypes = [vp, _f32p, i, C.POINTER(f), _f32p]
    L.rtm_ae_train_step.argtypes = [vp, _f32p, i, f, C.POINTER(f)]
    L.rtm_ae_reconstruct.argtypes = [vp, _f32p, i, _f32p, _f32p]
    L.rtm_ae_compress_volume.argtypes = [vp, vp, i, i, i, vp, vp, vp]
    L.rtm_ae_decompress_volume.argtypes = [vp, vp, vp, i, i, i, vp, vp]
    L.rtm_set_compressor.argtypes = [vp, vp]
    L.rtm_last_loop_launches.argtypes = [vp, C.POINTER(C.c_longlong)]
    L.rtm_profile.argtypes = [vp, i]
    L.rtm_profile_read.argtypes = [vp, np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"),
                                   np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")]
    for name in EXPORTS:
        fn = getattr(L, name)
        if name not in ("rtm_config_default", "rtm_last_error"):
            fn.restype = C.c_int
    _lib = L
    return L


def check(code, what, handle=None):
    if code != RTM_OK:
        detail = lib().rtm_last_error(handle)
        raise RtmError(code, what, detail.decode() if detail else "")
