"""libprofit's Model / Profile API in Python, backed by the sm_100a library.

Mirrors profit::Model (src/libprofit/src/profit/model.h:55-421) and
profit::Profile::parameter (profile.h:150-177): same method names, the same
parameter names and types, and the same errors (InvalidParameter for
profit::invalid_parameter, UnknownParameter for profit::unknown_parameter).
Images are numpy arrays of shape (height, width); pixel (x, y) is
image[y, x], which is libprofit's x-fastest row-major layout.
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

from . import _capi
from ._capi import PF_FP32, PF_FP64, check, lib, pf_param_ref

BOOL_PARAMS = {"rough", "adjust", "force_cpu", "convolve", "rescale_flux"}
UINT_PARAMS = {"resolution", "max_recursions"}


class Profile:
    """A profile added to a Model (profit::Profile)."""

    def __init__(self, model: "Model", index: int, name: str):
        self.model = model
        self.index = index
        self.name = name

    def parameter(self, name: str, value=None) -> "Profile":
        """Profile::parameter(name, value) or Profile::parameter("name = value")."""
        L, h = lib(), self.model._h
        if value is None:
            check(L.pf_profile_set(h, self.index, name.encode()))
        elif name in BOOL_PARAMS or isinstance(value, (bool, np.bool_)):
            check(L.pf_profile_set_bool(h, self.index, name.encode(), int(bool(value))))
        elif name in UINT_PARAMS:
            check(L.pf_profile_set_uint(h, self.index, name.encode(), int(value)))
        else:
            check(L.pf_profile_set_double(h, self.index, name.encode(), float(value)))
        return self

    def get(self, name: str) -> float:
        v = C.c_double()
        check(lib().pf_profile_get_double(self.model._h, self.index, name.encode(), C.byref(v)))
        return v.value

    def __setitem__(self, name, value):
        self.parameter(name, value)

    def __getitem__(self, name):
        return self.get(name)


class Model:
    """profit::Model on a B200.  One handle per host thread."""

    def __init__(self, width: int, height: int, precision: int = PF_FP64):
        h = C.c_void_p()
        check(lib().pf_model_create(int(width), int(height), C.byref(h)))
        self._h = h
        self.width, self.height = int(width), int(height)
        self.profiles: List[Profile] = []
        if precision != PF_FP64:
            self.set_precision(precision)

    def close(self):
        if getattr(self, "_h", None):
            lib().pf_model_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- profiles -------------------------------------------------------
    def add_profile(self, name: str, **params) -> Profile:
        idx = C.c_int()
        check(lib().pf_model_add_profile(self._h, name.encode(), C.byref(idx)))
        p = Profile(self, idx.value, name)
        self.profiles.append(p)
        for k, v in params.items():
            p.parameter(k, v)
        return p

    def clear_profiles(self):
        check(lib().pf_model_clear_profiles(self._h))
        self.profiles = []

    # --- settings (model.h:142-343) --------------------------------------
    def set_psf(self, psf: Optional[np.ndarray]):
        if psf is None:
            check(lib().pf_model_set_psf(self._h, None, 0, 0))
            return
        a = np.ascontiguousarray(psf, dtype=np.float64)
        h, w = a.shape
        check(lib().pf_model_set_psf(self._h, a.ctypes.data_as(_capi._dp), w, h))

    def set_magzero(self, magzero: float):
        check(lib().pf_model_set_magzero(self._h, float(magzero)))

    def set_image_pixel_scale(self, sx: float, sy: float):
        check(lib().pf_model_set_image_pixel_scale(self._h, float(sx), float(sy)))

    def set_psf_pixel_scale(self, sx: float, sy: float):
        check(lib().pf_model_set_psf_pixel_scale(self._h, float(sx), float(sy)))

    def set_finesampling(self, fs: int):
        check(lib().pf_model_set_finesampling(self._h, int(fs)))

    def set_return_finesampled(self, value: bool):
        check(lib().pf_model_set_return_finesampled(self._h, int(bool(value))))

    def set_crop(self, value: bool):
        check(lib().pf_model_set_crop(self._h, int(bool(value))))

    def set_convolver(self, kind: str):
        check(lib().pf_model_set_convolver(self._h, kind.encode()))

    def set_precision(self, precision: int):
        check(lib().pf_model_set_precision(self._h, int(precision)))

    def set_mask(self, mask: Optional[np.ndarray], adjust: bool = True):
        """Model::set_mask and set_adjust_mask: mask[height, width], nonzero = compute."""
        L = lib()
        if mask is None:
            check(L.pf_model_set_mask(self._h, None, 0, 0))
        else:
            mk = np.ascontiguousarray(mask, dtype=np.uint8)
            self._mask = mk
            h, w = mk.shape
            check(L.pf_model_set_mask(self._h, mk.ctypes.data_as(C.POINTER(C.c_uint8)), w, h))
        check(L.pf_model_set_adjust_mask(self._h, int(bool(adjust))))

    def set_dimensions(self, width: int, height: int):
        check(lib().pf_model_set_dimensions(self._h, int(width), int(height)))

    def set_dry_run(self, value: bool):
        check(lib().pf_model_set_dry_run(self._h, int(bool(value))))

    def set_omp_threads(self, n: int):
        """Accepted for libprofit compatibility; no effect (the work runs on the GPU)."""
        check(lib().pf_model_set_omp_threads(self._h, int(n)))

    def benchmark_convolvers(self, nbench: int = 10):
        """profitSetupData's benchmarked convolver choice: times "brute" and
        "fft" on this model as set up, keeps the faster one and returns
        (name, {"brute": ms, "fft": ms}) (mean device times; -1: not applicable)."""
        buf = C.create_string_buffer(16)
        tb, tf = C.c_double(), C.c_double()
        check(lib().pf_model_benchmark_convolvers(self._h, int(nbench), buf, 16, C.byref(tb), C.byref(tf)))
        return buf.value.decode(), {"brute": tb.value, "fft": tf.value}

    def set_likelihood(self, name: str):
        """profitLikeModel's like.func: "norm", "chisq", "t" or "pois" (and their aliases)."""
        check(lib().pf_model_set_likelihood(self._h, name.encode()))

    def set_adjoint_mode(self, mode: int):
        """PF_ADJOINT_AUTO / PF_ADJOINT_STORE / PF_ADJOINT_RECOMPUTE (see profit_b200.h)."""
        check(lib().pf_model_set_adjoint_mode(self._h, int(mode)))

    def set_debug(self, value: bool):
        check(lib().pf_model_set_debug(self._h, int(bool(value))))

    def drawing_dims(self) -> Tuple[int, int]:
        w, h = C.c_uint(), C.c_uint()
        check(lib().pf_model_drawing_dims(self._h, C.byref(w), C.byref(h)))
        return w.value, h.value

    # --- evaluation -------------------------------------------------------
    def evaluate(self) -> Tuple[np.ndarray, Tuple[int, int]]:
        """Model::evaluate: (image[height, width], (offset_x, offset_y))."""
        dw, dh = self.drawing_dims()
        cap = dw * dh
        buf = np.empty(cap, dtype=np.float64)
        w, h, ox, oy = C.c_uint(), C.c_uint(), C.c_int(), C.c_int()
        check(lib().pf_model_evaluate(self._h, buf.ctypes.data_as(_capi._dp), cap, C.byref(w), C.byref(h),
                                      C.byref(ox), C.byref(oy)))
        return buf[: w.value * h.value].reshape(h.value, w.value).copy(), (ox.value, oy.value)

    def set_data(self, image: np.ndarray, sigma: np.ndarray, region: Optional[np.ndarray] = None):
        im = np.ascontiguousarray(image, dtype=np.float64)
        sg = np.ascontiguousarray(sigma, dtype=np.float64)
        if sg.shape != im.shape:
            raise ValueError("sigma must have the image's shape")
        rp = None
        if region is not None:
            rg = np.ascontiguousarray(region, dtype=np.uint8)
            self._region = rg
            rp = rg.ctypes.data_as(C.POINTER(C.c_uint8))
        h, w = im.shape
        check(lib().pf_model_set_data(self._h, im.ctypes.data_as(_capi._dp), sg.ctypes.data_as(_capi._dp), rp, w, h))

    def loglike(self) -> float:
        v = C.c_double()
        check(lib().pf_model_loglike(self._h, C.byref(v)))
        return v.value

    @staticmethod
    def _refs(params: Sequence[Tuple[int, str]]):
        arr = (pf_param_ref * max(len(params), 1))()
        keep = []
        for i, (p, name) in enumerate(params):
            b = name.encode()
            keep.append(b)
            arr[i].profile = int(p.index if isinstance(p, Profile) else p)
            arr[i].name = b
        return arr, keep

    def set_parameters(self, params: Sequence[Tuple[int, str]], values: Sequence[float]):
        """Writes a whole parameter vector in one call (a sampler's next proposal)."""
        arr, keep = self._refs(params)
        v = np.ascontiguousarray(values, dtype=np.float64)
        check(lib().pf_model_set_parameters(self._h, arr, len(params), v.ctypes.data_as(_capi._dp)))

    def loglike_grad(self, params: Sequence[Tuple[int, str]]) -> Tuple[float, np.ndarray]:
        """logL and its adjoint gradient (FP32 path)."""
        arr, keep = self._refs(params)
        ll = C.c_double()
        g = np.zeros(len(params), dtype=np.float64)
        check(lib().pf_model_loglike_grad(self._h, arr, len(params), C.byref(ll), g.ctypes.data_as(_capi._dp)))
        return ll.value, g

    def loglike_grad_batch(self, params: Sequence[Tuple[int, str]], values: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        """logL[b] and gradient[b, i] for every row of values[b, i] (a batch of proposals).
        Invalid proposals get logL = -inf."""
        arr, keep = self._refs(params)
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1, len(params))
        B = v.shape[0]
        ll = np.zeros(B, dtype=np.float64)
        g = np.zeros((B, len(params)), dtype=np.float64)
        check(lib().pf_model_loglike_grad_batch(self._h, arr, len(params), B, v.ctypes.data_as(_capi._dp),
                                                ll.ctypes.data_as(_capi._dp), g.ctypes.data_as(_capi._dp)))
        return ll, g

    def set_fit_space(self, params: Sequence[Tuple[int, str]], init: Sequence[float],
                      tofit: Sequence[Optional[bool]], tolog: Optional[Sequence[bool]] = None,
                      intervals: Optional[Sequence[Optional[Tuple[float, float]]]] = None,
                      offset: Optional[Sequence[float]] = None, prior_sigmas: Optional[Sequence[float]] = None,
                      prior_means: Optional[Sequence[float]] = None, prior_tolog: Optional[Sequence[bool]] = None,
                      prior_on: Optional[Sequence[bool]] = None):
        """Installs ProFit's fit space on the model (pf_model_set_fit_space):
        entries in unlist(modellist) order; tofit True / False / None (R's NA:
        the value of the entry before); intervals (lo, hi) or None per entry;
        offset (x, y, ang, size) with NaN for R's NA; normal priors with an
        infinite sigma for a flat one, on every entry unless prior_on says."""
        n = len(params)
        arr, keep = self._refs(params)
        d = lambda v: np.ascontiguousarray(v, dtype=np.float64)  # noqa: E731
        ints = lambda v: None if v is None else (C.c_int * n)(*[int(bool(x)) for x in v])  # noqa: E731
        init_a = d(init)
        fit_a = (C.c_int * n)(*[-1 if f is None else int(bool(f)) for f in tofit])
        lo = hi = None
        if intervals is not None:
            lo = d([np.nan if iv is None else iv[0] for iv in intervals])
            hi = d([np.nan if iv is None else iv[1] for iv in intervals])
        off = None if offset is None else d(offset)
        sig = None if prior_sigmas is None else d(prior_sigmas)
        mean = None if prior_means is None else d(prior_means)
        self._fit_keep = (keep, init_a, lo, hi, off, sig, mean)
        p = lambda a: None if a is None else a.ctypes.data_as(_capi._dp)  # noqa: E731
        check(lib().pf_model_set_fit_space(self._h, n, arr, p(init_a), fit_a, ints(tolog), p(lo), p(hi), p(off), p(sig),
                                           p(mean), ints(prior_tolog), ints(prior_on)))

    def fit_size(self) -> Tuple[int, int]:
        """(number of fitted entries, number of entries) of the fit space."""
        nf, ne = C.c_int(), C.c_int()
        check(lib().pf_model_fit_size(self._h, C.byref(nf), C.byref(ne)))
        return nf.value, ne.value

    def lp_grad_batch(self, parm: np.ndarray) -> Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]:
        """LP = LL + log prior, d LP / d parm, parm_out (limits applied, as
        profitRemakeModellist returns it) and LL for every row of parm[b, j]."""
        nf, _ = self.fit_size()
        v = np.ascontiguousarray(parm, dtype=np.float64).reshape(-1, nf)
        B = v.shape[0]
        lp = np.zeros(B)
        g = np.zeros((B, nf))
        out = np.zeros((B, nf))
        ll = np.zeros(B)
        P = _capi._dp
        check(lib().pf_model_lp_grad_batch(self._h, B, v.ctypes.data_as(P), lp.ctypes.data_as(P), g.ctypes.data_as(P),
                                           out.ctypes.data_as(P), ll.ctypes.data_as(P)))
        return lp, g, out, ll

    def loglike_grad_fd(self, params: Sequence[Tuple[int, str]], rel_step: float = 1e-6) -> Tuple[float, np.ndarray]:
        """logL and central finite differences of the plain FP64 form."""
        arr, keep = self._refs(params)
        ll = C.c_double()
        g = np.zeros(len(params), dtype=np.float64)
        check(lib().pf_model_loglike_grad_fd(self._h, arr, len(params), float(rel_step), C.byref(ll),
                                             g.ctypes.data_as(_capi._dp)))
        return ll.value, g

    # --- instrumentation ---------------------------------------------------
    def decisions(self, profile: int) -> np.ndarray:
        dw, dh = self.drawing_dims()
        out = np.zeros(dw * dh, dtype=np.int32)
        check(lib().pf_model_decisions(self._h, int(profile), out.ctypes.data_as(C.POINTER(C.c_int32)), out.size))
        return out.reshape(dh, dw)

    def level_counts(self, profile: int) -> List[int]:
        out = (C.c_int64 * 16)()
        n = C.c_int()
        check(lib().pf_model_level_counts(self._h, int(profile), out, 16, C.byref(n)))
        return [out[i] for i in range(n.value)]

    def evaluation_counts(self, profile: int) -> Tuple[int, List[int]]:
        """Profile evaluations of the last debug evaluation: (total, [direct,
        level 0, level 1, ...]) with trailing empty levels dropped."""
        out = (C.c_int64 * 17)()
        tot = C.c_int64()
        check(lib().pf_model_evaluation_counts(self._h, int(profile), out, 17, C.byref(tot)))
        per = [out[i] for i in range(17)]
        while len(per) > 1 and per[-1] == 0:
            per.pop()
        return tot.value, per

    def last_timings(self) -> List[float]:
        """Device ms of the last evaluation: [total, render, convolution,
        likelihood + adjoint]; the phases are NaN for a replayed FP32
        pipeline unless set_phase_timing(True)."""
        out = (C.c_float * 4)()
        check(lib().pf_model_last_timings(self._h, out, 4))
        return list(out)

    def set_phase_timing(self, on: bool = True) -> None:
        """Records the phase events inside replayed FP32 pipelines (a few
        microseconds of device time per replay)."""
        check(lib().pf_model_set_phase_timing(self._h, int(bool(on))))
