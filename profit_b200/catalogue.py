"""Catalogue batches: many galaxies, each with its own image, sigma map, PSF and
profiles, evaluated for logL and gradient in one call (pf_catalogue_* in the C
ABI).  There is no libprofit counterpart; ProFit fits one galaxy per
profitLikeModel call, and this is the same computation for a whole list."""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import _capi
from ._capi import check, lib

# d logL / d(...) order for one profile: these six, then the kind's shape parameters.
COMMON_GRAD = ("xcen", "ycen", "mag", "ang", "axrat", "box")
SHAPE_GRAD = {
    "sersic": ("re", "nser"),
    "moffat": ("fwhm", "con"),
    "ferrer": ("rout", "a", "b"),
    "coresersic": ("re", "rb", "nser", "a", "b"),
    "king": ("rc", "rt", "a"),
    "brokenexp": ("h1", "h2", "rb", "a"),
}


def grad_names(kind: str) -> Tuple[str, ...]:
    return COMMON_GRAD + SHAPE_GRAD[kind]


class Catalogue:
    def __init__(self, magzero: float = 0.0):
        h = C.c_void_p()
        check(lib().pf_catalogue_create(C.byref(h)))
        self._h = h
        self._kinds: List[List[str]] = []
        check(lib().pf_catalogue_set_magzero(self._h, float(magzero)))

    def close(self):
        if getattr(self, "_h", None):
            lib().pf_catalogue_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_galaxy(self, data: np.ndarray, sigma: np.ndarray, psf: np.ndarray,
                   profiles: Sequence[Tuple[str, Dict[str, float]]]) -> int:
        d = np.ascontiguousarray(data, dtype=np.float64)
        s = np.ascontiguousarray(sigma, dtype=np.float64)
        p = np.ascontiguousarray(psf, dtype=np.float64)
        if s.shape != d.shape:
            raise ValueError("sigma must have the image's shape")
        h, w = d.shape
        ph, pw = p.shape
        idx = C.c_int()
        check(lib().pf_catalogue_add_galaxy(self._h, w, h, d.ctypes.data_as(_capi._dp), s.ctypes.data_as(_capi._dp),
                                            p.ctypes.data_as(_capi._dp), pw, ph, C.byref(idx)))
        kinds = []
        for kind, params in profiles:
            names = [k.encode() for k in params]
            vals = np.array([float(v) for v in params.values()], dtype=np.float64)
            arr = (C.c_char_p * max(len(names), 1))(*names)
            check(lib().pf_catalogue_add_profile(self._h, idx.value, kind.encode(), len(names), arr,
                                                 vals.ctypes.data_as(_capi._dp)))
            kinds.append(kind)
        self._kinds.append(kinds)
        return idx.value

    def size(self) -> Tuple[int, int]:
        n, g = C.c_int(), C.c_int()
        check(lib().pf_catalogue_size(self._h, C.byref(n), C.byref(g)))
        return n.value, g.value

    def loglike_grad(self) -> Tuple[np.ndarray, List[np.ndarray]]:
        """logL per galaxy and, per galaxy, its gradient vector (profile after
        profile in grad_names(kind) order)."""
        n, ng = self.size()
        ll = np.zeros(n)
        g = np.zeros(max(ng, 1))
        check(lib().pf_catalogue_loglike_grad(self._h, ll.ctypes.data_as(_capi._dp), g.ctypes.data_as(_capi._dp)))
        out, off = [], 0
        for kinds in self._kinds:
            k = sum(len(grad_names(kd)) for kd in kinds)
            out.append(g[off:off + k].copy())
            off += k
        return ll, out

    def values(self) -> np.ndarray:
        """Every profile's parameters in the gradient's layout (galaxy after
        galaxy, profile after profile, grad_names(kind) order)."""
        _, ng = self.size()
        v = np.zeros(max(ng, 1))
        check(lib().pf_catalogue_get_values(self._h, v.ctypes.data_as(_capi._dp)))
        return v[:ng]

    def set_values(self, values) -> None:
        """New parameters for every profile (the layout of values()); the
        next loglike_grad keeps the images, batching and recorded launches."""
        _, ng = self.size()
        v = np.ascontiguousarray(values, dtype=np.float64)
        if v.shape != (ng,):
            raise ValueError(f"expected {ng} values, got shape {v.shape}")
        check(lib().pf_catalogue_set_values(self._h, v.ctypes.data_as(_capi._dp)))

    def set_convolver(self, name: str) -> None:
        """"auto" (each batch of galaxies keeps the faster of brute force and
        FP64 FFTs, timed once), "brute" or "fft"."""
        check(lib().pf_catalogue_set_convolver(self._h, name.encode()))

    def convolvers(self) -> Tuple[int, int]:
        """(batches convolved through FFTs, batches), after an evaluation."""
        f, n = C.c_int(), C.c_int()
        check(lib().pf_catalogue_convolvers(self._h, C.byref(f), C.byref(n)))
        return f.value, n.value

    def last_time_ms(self) -> float:
        t = C.c_float()
        check(lib().pf_catalogue_last_time(self._h, C.byref(t)))
        return t.value
