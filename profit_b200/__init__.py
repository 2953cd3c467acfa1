"""profit_b200: ProFit / libprofit model images and likelihoods on B200 (sm_100a).

The compute path is the C-ABI library profit_b200/lib/libprofit_b200.so
(hand-written CUDA); this package is its Python binding with libprofit's
Model/Profile API.
"""
from ._capi import (PF_FP32, PF_FP32_CONV64, PF_FP64, InvalidParameter, ProfitError, UnknownParameter, LIB_PATH, EXPORTED)
from .model import Model, Profile

__all__ = ["Model", "Profile", "PF_FP32", "PF_FP32_CONV64", "PF_FP64", "ProfitError", "InvalidParameter", "UnknownParameter",
           "LIB_PATH", "EXPORTED"]
