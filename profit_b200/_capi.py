"""ctypes binding of the C ABI in include/profit_b200.h.

The shared library is built in-tree (profit_b200/lib/libprofit_b200.so) by
profit_b200.build; importing this module never falls back to anything else:
if the library is missing or no B200 is present, calls fail with ProfitError.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libprofit_b200.so")

PF_OK = 0
PF_E_INVALID = -1
PF_E_UNKNOWN_PARAM = -2
PF_E_CUDA = -3
PF_E_CAPACITY = -4
PF_E_BUFFER = -5
PF_E_STATE = -6
PF_FP64 = 0
PF_FP32 = 1
PF_FP32_CONV64 = 2

# Every symbol include/profit_b200.h declares.
EXPORTED = (
    "pf_last_error", "pf_version", "pf_model_create", "pf_model_destroy", "pf_model_add_profile",
    "pf_profile_set_double", "pf_profile_set_uint", "pf_profile_set_bool", "pf_profile_set",
    "pf_profile_get_double", "pf_model_profile_count", "pf_model_clear_profiles", "pf_model_set_psf",
    "pf_model_set_magzero", "pf_model_set_image_pixel_scale", "pf_model_set_psf_pixel_scale",
    "pf_model_set_finesampling", "pf_model_set_return_finesampled", "pf_model_set_crop",
    "pf_model_set_convolver", "pf_model_set_precision", "pf_model_drawing_dims", "pf_model_evaluate",
    "pf_model_set_data", "pf_model_loglike", "pf_model_loglike_grad", "pf_model_loglike_grad_fd",
    "pf_model_set_debug", "pf_model_decisions", "pf_model_level_counts", "pf_model_evaluation_counts", "pf_model_last_timings",
    "pf_model_set_phase_timing",
    "pf_kernel_launches",
)


class ProfitError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class InvalidParameter(ProfitError):
    pass


class UnknownParameter(InvalidParameter):
    pass


class pf_param_ref(C.Structure):
    _fields_ = [("profile", C.c_int), ("name", C.c_char_p)]


_lib = None
_lock = threading.Lock()
_dp = C.POINTER(C.c_double)


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: build it with `python -m profit_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.pf_last_error.restype = C.c_char_p
        L.pf_version.restype = C.c_char_p
        L.pf_model_create.argtypes = [C.c_uint, C.c_uint, C.POINTER(vp)]
        L.pf_model_destroy.argtypes = [vp]
        L.pf_model_add_profile.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int)]
        L.pf_profile_set_double.argtypes = [vp, C.c_int, C.c_char_p, C.c_double]
        L.pf_profile_set_uint.argtypes = [vp, C.c_int, C.c_char_p, C.c_uint]
        L.pf_profile_set_bool.argtypes = [vp, C.c_int, C.c_char_p, C.c_int]
        L.pf_profile_set.argtypes = [vp, C.c_int, C.c_char_p]
        L.pf_profile_get_double.argtypes = [vp, C.c_int, C.c_char_p, _dp]
        L.pf_model_profile_count.argtypes = [vp, C.POINTER(C.c_int)]
        L.pf_model_clear_profiles.argtypes = [vp]
        L.pf_model_set_psf.argtypes = [vp, _dp, C.c_uint, C.c_uint]
        L.pf_model_set_magzero.argtypes = [vp, C.c_double]
        L.pf_model_set_image_pixel_scale.argtypes = [vp, C.c_double, C.c_double]
        L.pf_model_set_psf_pixel_scale.argtypes = [vp, C.c_double, C.c_double]
        L.pf_model_set_finesampling.argtypes = [vp, C.c_uint]
        L.pf_model_set_return_finesampled.argtypes = [vp, C.c_int]
        L.pf_model_set_crop.argtypes = [vp, C.c_int]
        L.pf_model_set_convolver.argtypes = [vp, C.c_char_p]
        L.pf_model_set_precision.argtypes = [vp, C.c_int]
        L.pf_model_drawing_dims.argtypes = [vp, C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
        L.pf_model_evaluate.argtypes = [vp, _dp, C.c_size_t, C.POINTER(C.c_uint), C.POINTER(C.c_uint),
                                        C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.pf_model_set_data.argtypes = [vp, _dp, _dp, C.POINTER(C.c_uint8), C.c_uint, C.c_uint]
        L.pf_model_loglike.argtypes = [vp, _dp]
        L.pf_model_loglike_grad.argtypes = [vp, C.POINTER(pf_param_ref), C.c_int, _dp, _dp]
        L.pf_model_loglike_grad_fd.argtypes = [vp, C.POINTER(pf_param_ref), C.c_int, C.c_double, _dp, _dp]
        L.pf_model_set_debug.argtypes = [vp, C.c_int]
        L.pf_model_set_phase_timing.argtypes = [vp, C.c_int]
        L.pf_model_decisions.argtypes = [vp, C.c_int, C.POINTER(C.c_int32), C.c_size_t]
        L.pf_model_level_counts.argtypes = [vp, C.c_int, C.POINTER(C.c_int64), C.c_int, C.POINTER(C.c_int)]
        L.pf_model_evaluation_counts.argtypes = [vp, C.c_int, C.POINTER(C.c_int64), C.c_int, C.POINTER(C.c_int64)]
        L.pf_model_last_timings.argtypes = [vp, C.POINTER(C.c_float), C.c_int]
        L.pf_kernel_launches.restype = C.c_ulonglong
        _late_bindings(L)
        _lib = L
    return _lib


def check(status: int) -> None:
    if status == PF_OK:
        return
    msg = lib().pf_last_error().decode()
    if status == PF_E_UNKNOWN_PARAM:
        raise UnknownParameter(status, msg)
    if status == PF_E_INVALID:
        raise InvalidParameter(status, msg)
    raise ProfitError(status, msg)


def _late_bindings(L):
    L.pf_model_set_parameters.argtypes = [C.c_void_p, C.POINTER(pf_param_ref), C.c_int, _dp]
    L.pf_model_loglike_grad_batch.argtypes = [C.c_void_p, C.POINTER(pf_param_ref), C.c_int, C.c_int, _dp, _dp, _dp]
    L.pf_model_set_adjoint_mode.argtypes = [C.c_void_p, C.c_int]
    L.pf_model_set_likelihood.argtypes = [C.c_void_p, C.c_char_p]
    L.pf_model_set_mask.argtypes = [C.c_void_p, C.POINTER(C.c_uint8), C.c_uint, C.c_uint]
    L.pf_model_set_adjust_mask.argtypes = [C.c_void_p, C.c_int]
    L.pf_model_set_dimensions.argtypes = [C.c_void_p, C.c_uint, C.c_uint]
    L.pf_model_set_dry_run.argtypes = [C.c_void_p, C.c_int]
    L.pf_model_set_omp_threads.argtypes = [C.c_void_p, C.c_uint]
    L.pf_model_benchmark_convolvers.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_size_t, _dp, _dp]
    vp = C.c_void_p
    L.pf_catalogue_create.argtypes = [C.POINTER(vp)]
    L.pf_catalogue_destroy.argtypes = [vp]
    L.pf_catalogue_set_magzero.argtypes = [vp, C.c_double]
    L.pf_catalogue_add_galaxy.argtypes = [vp, C.c_uint, C.c_uint, _dp, _dp, _dp, C.c_uint, C.c_uint,
                                          C.POINTER(C.c_int)]
    L.pf_catalogue_add_profile.argtypes = [vp, C.c_int, C.c_char_p, C.c_int, C.POINTER(C.c_char_p), _dp]
    L.pf_catalogue_size.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.pf_catalogue_gradient_offset.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.pf_catalogue_loglike_grad.argtypes = [vp, _dp, _dp]
    L.pf_catalogue_last_time.argtypes = [vp, C.POINTER(C.c_float)]
    L.pf_catalogue_set_values.argtypes = [vp, _dp]
    L.pf_catalogue_get_values.argtypes = [vp, _dp]
    L.pf_catalogue_set_convolver.argtypes = [vp, C.c_char_p]
    L.pf_catalogue_convolvers.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    ip = C.POINTER(C.c_int)
    L.pf_model_set_fit_space.argtypes = [vp, C.c_int, C.POINTER(pf_param_ref), _dp, ip, ip, _dp, _dp, _dp, _dp, _dp,
                                         ip, ip]
    L.pf_model_fit_size.argtypes = [vp, ip, ip]
    L.pf_model_lp_grad_batch.argtypes = [vp, C.c_int, _dp, _dp, _dp, _dp, _dp]
    # device pointers travel as plain integers (e.g. a torch tensor's data_ptr())
    L.pf_loglike_norm_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_int,
                                          C.c_void_p, C.c_void_p]


PF_ADJOINT_AUTO = 0
PF_ADJOINT_STORE = 1
PF_ADJOINT_RECOMPUTE = 2
PF_LOGLIKE_NOALLOC_MAX_BATCH = 64

EXPORTED = EXPORTED + ("pf_model_set_parameters", "pf_model_loglike_grad_batch", "pf_model_set_adjoint_mode",
                       "pf_loglike_norm_noalloc", "pf_catalogue_create", "pf_catalogue_destroy",
                       "pf_catalogue_set_magzero", "pf_catalogue_add_galaxy", "pf_catalogue_add_profile",
                       "pf_catalogue_size", "pf_catalogue_gradient_offset", "pf_catalogue_loglike_grad",
                       "pf_catalogue_last_time", "pf_catalogue_set_values", "pf_catalogue_get_values",
                       "pf_catalogue_set_convolver", "pf_catalogue_convolvers",
                       "pf_model_set_likelihood", "pf_model_set_mask",
                       "pf_model_set_adjust_mask", "pf_model_set_dimensions", "pf_model_set_dry_run",
                       "pf_model_set_omp_threads", "pf_model_benchmark_convolvers", "pf_model_set_fit_space",
                       "pf_model_fit_size", "pf_model_lp_grad_batch")
