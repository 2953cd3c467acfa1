"""ORACLE (test infrastructure only): ctypes access to the two CPU checkers.

* ``RefModel`` drives the reference's own libprofit C++ compiled in place by
  ``oracle/Makefile`` (``oracle/_ref/libprofit_ref.so``): profit::Model
  (src/libprofit/src/profit/model.h:55-421) behind ``oracle/ref_harness.cpp``.
* ``OracleModel`` drives the plain-C restatement ``oracle/profit_oracle.c``
  (``oracle/_build/liboracle.so``), which also logs per-pixel subsampling
  decisions and restates the likelihood of R/profitLikeModel.R:263-276.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Iterable, Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libprofit_ref.so")
REF_DBG_SO = os.path.join(HERE, "_ref", "libprofit_ref_dbg.so")
# Speed builds of the same sources for the timed CPU baseline (oracle/Makefile):
# ISA level -> library, and the /proc/cpuinfo flags each level needs.
REF_FAST_SO = {
    "x86-64-v4": os.path.join(HERE, "_ref", "libprofit_ref_v4.so"),
    "x86-64-v3": os.path.join(HERE, "_ref", "libprofit_ref_v3.so"),
}
_ISA_FLAGS = {
    "x86-64-v3": {"avx", "avx2", "bmi1", "bmi2", "f16c", "fma", "abm", "movbe", "xsave"},
    "x86-64-v4": {"avx", "avx2", "bmi1", "bmi2", "f16c", "fma", "abm", "movbe", "xsave",
                  "avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"},
}
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")

_dp = C.POINTER(C.c_double)

# Parameter types of every libprofit profile (profile.h register_parameter
# calls in radial.cpp:738-751, sersic.cpp:356-358, moffat.cpp:103-104, ...).
BOOL_PARAMS = {"rough", "adjust", "force_cpu", "convolve", "rescale_flux"}
UINT_PARAMS = {"resolution", "max_recursions"}


def _load(path: str) -> C.CDLL:
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
    return C.CDLL(path)


class _RefLib:
    _libs: Dict[str, C.CDLL] = {}

    @classmethod
    def get(cls, debug: bool = False, build: str = "parity") -> C.CDLL:
        path = REF_DBG_SO if debug else (REF_SO if build == "parity" else REF_FAST_SO[build])
        if path not in cls._libs:
            lib = _load(path)
            lib.pfref_model_new.restype = C.c_void_p
            lib.pfref_model_new.argtypes = [C.c_uint, C.c_uint]
            lib.pfref_model_free.argtypes = [C.c_void_p]
            lib.pfref_add_profile.argtypes = [C.c_void_p, C.c_char_p]
            lib.pfref_profile_set_double.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_double]
            lib.pfref_profile_set_uint.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_uint]
            lib.pfref_profile_set_bool.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_int]
            lib.pfref_profile_set.argtypes = [C.c_void_p, C.c_int, C.c_char_p]
            lib.pfref_set_psf.argtypes = [C.c_void_p, _dp, C.c_uint, C.c_uint]
            lib.pfref_set_magzero.argtypes = [C.c_void_p, C.c_double]
            lib.pfref_set_scale.argtypes = [C.c_void_p, C.c_double, C.c_double]
            lib.pfref_set_psf_scale.argtypes = [C.c_void_p, C.c_double, C.c_double]
            lib.pfref_set_finesampling.argtypes = [C.c_void_p, C.c_uint]
            lib.pfref_set_return_finesampled.argtypes = [C.c_void_p, C.c_int]
            lib.pfref_set_crop.argtypes = [C.c_void_p, C.c_int]
            lib.pfref_set_omp_threads.argtypes = [C.c_void_p, C.c_uint]
            lib.pfref_set_adjust_mask.argtypes = [C.c_void_p, C.c_int]
            lib.pfref_set_mask.argtypes = [C.c_void_p, C.POINTER(C.c_uint8), C.c_uint, C.c_uint]
            lib.pfref_set_convolver.argtypes = [C.c_void_p, C.c_char_p, C.c_uint]
            lib.pfref_drawing_dims.argtypes = [C.c_void_p, C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
            lib.pfref_evaluate.argtypes = [C.c_void_p, _dp, C.c_size_t, C.POINTER(C.c_uint),
                                           C.POINTER(C.c_uint), C.POINTER(C.c_int), C.POINTER(C.c_int)]
            lib.pfref_last_error.restype = C.c_char_p
            for fn in ("pfref_qgamma", "pfref_pgamma", "pfref_beta"):
                getattr(lib, fn).restype = C.c_double
                getattr(lib, fn).argtypes = [C.c_double, C.c_double]
            lib.pfref_gammafn.restype = C.c_double
            lib.pfref_gammafn.argtypes = [C.c_double]
            integrand = C.CFUNCTYPE(C.c_double, C.c_double, C.c_void_p)
            lib._integrand_t = integrand
            lib.pfref_integrate_qags.restype = C.c_double
            lib.pfref_integrate_qags.argtypes = [integrand, C.c_void_p, C.c_double, C.c_double]
            lib.pfref_integrate_qagi.restype = C.c_double
            lib.pfref_integrate_qagi.argtypes = [integrand, C.c_void_p, C.c_double]
            if debug:
                lib.pfref_integrations.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_int]
            cls._libs[path] = lib
        return cls._libs[path]


class RefError(RuntimeError):
    pass


def host_cpu_flags() -> set:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def runnable_reference_builds() -> list:
    """The builds of the reference this host can run: the speed builds whose
    ISA level the CPU supports (highest first), then the parity build."""
    flags = host_cpu_flags()
    out = [b for b in ("x86-64-v4", "x86-64-v3")
           if _ISA_FLAGS[b] <= flags and os.path.exists(REF_FAST_SO[b])]
    return out + ["parity"]


class RefModel:
    """profit::Model from the compiled reference, configured like R_profit_make_model.

    build: "parity" (-O3 -mavx -ffp-contract=off, the build parity is pinned
    on), or a speed build "x86-64-v3" / "x86-64-v4" (-O3 -march=..., GNU
    mode) for timing; debug selects the PROFIT_DEBUG parity build."""

    def __init__(self, width: int, height: int, debug: bool = False, build: str = "parity"):
        self.lib = _RefLib.get(debug, build)
        self.debug = debug
        self.h = self.lib.pfref_model_new(width, height)
        self.nprof = 0

    def __del__(self):
        try:
            self.lib.pfref_model_free(self.h)
        except Exception:
            pass

    def _check(self, st: int):
        if st != 0:
            raise RefError(self.lib.pfref_last_error().decode())

    def add_profile(self, name: str, **params) -> int:
        idx = self.lib.pfref_add_profile(self.h, name.encode())
        if idx < 0:
            raise RefError(self.lib.pfref_last_error().decode())
        for k, v in params.items():
            self.set(idx, k, v)
        self.nprof += 1
        return idx

    def set(self, idx: int, name: str, value):
        b = name.encode()
        if name in BOOL_PARAMS:
            self._check(self.lib.pfref_profile_set_bool(self.h, idx, b, int(bool(value))))
        elif name in UINT_PARAMS:
            self._check(self.lib.pfref_profile_set_uint(self.h, idx, b, int(value)))
        else:
            self._check(self.lib.pfref_profile_set_double(self.h, idx, b, float(value)))

    def set_spec(self, idx: int, spec: str):
        self._check(self.lib.pfref_profile_set(self.h, idx, spec.encode()))

    def set_psf(self, psf: np.ndarray):
        psf = np.ascontiguousarray(psf, dtype=np.float64)
        h, w = psf.shape
        self._check(self.lib.pfref_set_psf(self.h, psf.ctypes.data_as(_dp), w, h))

    def set_magzero(self, mz: float):
        self.lib.pfref_set_magzero(self.h, mz)

    def set_scale(self, sx: float, sy: float):
        self.lib.pfref_set_scale(self.h, sx, sy)

    def set_psf_scale(self, sx: float, sy: float):
        self.lib.pfref_set_psf_scale(self.h, sx, sy)

    def set_finesampling(self, fs: int):
        self._check(self.lib.pfref_set_finesampling(self.h, fs))

    def set_return_finesampled(self, v: bool):
        self.lib.pfref_set_return_finesampled(self.h, int(v))

    def set_crop(self, v: bool):
        self.lib.pfref_set_crop(self.h, int(v))

    def set_omp_threads(self, n: int):
        self.lib.pfref_set_omp_threads(self.h, n)

    def set_convolver(self, kind: str = "brute", omp_threads: int = 1):
        self._check(self.lib.pfref_set_convolver(self.h, kind.encode(), omp_threads))

    def set_mask(self, mask: np.ndarray, adjust: bool = True):
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        h, w = m.shape
        self._check(self.lib.pfref_set_mask(self.h, m.ctypes.data_as(C.POINTER(C.c_uint8)), w, h))
        self.lib.pfref_set_adjust_mask(self.h, int(adjust))

    def drawing_dims(self) -> Tuple[int, int]:
        w, h = C.c_uint(), C.c_uint()
        self._check(self.lib.pfref_drawing_dims(self.h, C.byref(w), C.byref(h)))
        return w.value, h.value

    def evaluate(self) -> Tuple[np.ndarray, Tuple[int, int]]:
        """Returns (image[h, w] row-major with x fastest, (offset_x, offset_y))."""
        dw, dh = self.drawing_dims()
        cap = max(dw * dh, 1) * 4
        buf = np.zeros(cap, dtype=np.float64)
        w, h, ox, oy = C.c_uint(), C.c_uint(), C.c_int(), C.c_int()
        self._check(self.lib.pfref_evaluate(self.h, buf.ctypes.data_as(_dp), cap, C.byref(w),
                                            C.byref(h), C.byref(ox), C.byref(oy)))
        return buf[: w.value * h.value].reshape(h.value, w.value).copy(), (ox.value, oy.value)

    def integrations(self, idx: int, max_levels: int = 16) -> list:
        """Per-level subsample_pixel call counts of profile idx (debug build only)."""
        if not self.debug:
            raise RefError("integration counters need the PROFIT_DEBUG build")
        counts = (C.c_int * max_levels)()
        n = self.lib.pfref_integrations(self.h, idx, counts, max_levels)
        if n < 0:
            return []
        return [counts[i] for i in range(n)]


def ref_special():
    """The shimmed special functions exactly as libprofit calls them."""
    lib = _RefLib.get(False)
    return {
        "qgamma": lib.pfref_qgamma,
        "pgamma": lib.pfref_pgamma,
        "gammafn": lib.pfref_gammafn,
        "beta": lib.pfref_beta,
    }


def ref_integrate(f, a: float, b: Optional[float] = None) -> float:
    """libprofit's integrate_qags (b given) or integrate_qagi (to +inf)."""
    lib = _RefLib.get(False)
    cb = lib._integrand_t(lambda x, _ud: f(x))
    if b is None:
        return lib.pfref_integrate_qagi(cb, None, a)
    return lib.pfref_integrate_qags(cb, None, a, b)


class _OracleLib:
    lib: Optional[C.CDLL] = None

    @classmethod
    def get(cls) -> C.CDLL:
        if cls.lib is None:
            lib = _load(ORACLE_SO)
            lib.pfo_model_new.restype = C.c_void_p
            lib.pfo_model_new.argtypes = [C.c_uint, C.c_uint]
            lib.pfo_model_free.argtypes = [C.c_void_p]
            lib.pfo_last_error.restype = C.c_char_p
            lib.pfo_add_profile.argtypes = [C.c_void_p, C.c_char_p]
            lib.pfo_profile_set_double.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_double]
            lib.pfo_profile_set_uint.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_uint]
            lib.pfo_profile_set_bool.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.c_int]
            lib.pfo_set_psf.argtypes = [C.c_void_p, _dp, C.c_uint, C.c_uint]
            lib.pfo_set_magzero.argtypes = [C.c_void_p, C.c_double]
            lib.pfo_set_scale.argtypes = [C.c_void_p, C.c_double, C.c_double]
            lib.pfo_set_psf_scale.argtypes = [C.c_void_p, C.c_double, C.c_double]
            lib.pfo_set_finesampling.argtypes = [C.c_void_p, C.c_uint]
            lib.pfo_set_return_finesampled.argtypes = [C.c_void_p, C.c_int]
            lib.pfo_set_convolver.argtypes = [C.c_void_p, C.c_char_p]
            lib.pfo_set_threads.argtypes = [C.c_void_p, C.c_int]
            lib.pfo_drawing_dims.argtypes = [C.c_void_p, C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
            lib.pfo_evaluate.argtypes = [C.c_void_p, _dp, C.c_size_t, C.POINTER(C.c_uint),
                                         C.POINTER(C.c_uint), C.POINTER(C.c_int), C.POINTER(C.c_int)]
            lib.pfo_decisions.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_size_t]
            lib.pfo_level_counts.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_long), C.c_int]
            lib.pfo_evaluations.argtypes = [C.c_void_p, C.c_int]
            lib.pfo_evaluations.restype = C.c_long
            lib.pfo_profile_scalars.argtypes = [C.c_void_p, C.c_int, _dp, C.c_int]
            lib.pfo_loglike_norm.restype = C.c_double
            lib.pfo_loglike_norm.argtypes = [_dp, _dp, _dp, C.POINTER(C.c_uint8), C.c_size_t]
            cls.lib = lib
        return cls.lib


SCALAR_NAMES = ("rscale", "ie", "bn", "acc", "rscale_switch", "rscale_max", "resolution",
                "flux_scale", "cos_ang", "sin_ang", "lumtot", "rescale_factor")


class OracleModel:
    """The plain-C restatement, with the same configuration calls as RefModel."""

    def __init__(self, width: int, height: int, threads: int = 1):
        self.lib = _OracleLib.get()
        self.h = self.lib.pfo_model_new(width, height)
        self.lib.pfo_set_threads(self.h, threads)
        self.nprof = 0

    def __del__(self):
        try:
            self.lib.pfo_model_free(self.h)
        except Exception:
            pass

    def _check(self, st: int):
        if st < 0:
            raise RefError(self.lib.pfo_last_error().decode())

    def add_profile(self, name: str, **params) -> int:
        idx = self.lib.pfo_add_profile(self.h, name.encode())
        self._check(idx)
        for k, v in params.items():
            self.set(idx, k, v)
        self.nprof += 1
        return idx

    def set(self, idx: int, name: str, value):
        b = name.encode()
        if name in BOOL_PARAMS:
            self._check(self.lib.pfo_profile_set_bool(self.h, idx, b, int(bool(value))))
        elif name in UINT_PARAMS:
            self._check(self.lib.pfo_profile_set_uint(self.h, idx, b, int(value)))
        else:
            self._check(self.lib.pfo_profile_set_double(self.h, idx, b, float(value)))

    def set_psf(self, psf: np.ndarray):
        psf = np.ascontiguousarray(psf, dtype=np.float64)
        h, w = psf.shape
        self._check(self.lib.pfo_set_psf(self.h, psf.ctypes.data_as(_dp), w, h))

    def set_magzero(self, mz: float):
        self.lib.pfo_set_magzero(self.h, mz)

    def set_scale(self, sx: float, sy: float):
        self.lib.pfo_set_scale(self.h, sx, sy)

    def set_psf_scale(self, sx: float, sy: float):
        self.lib.pfo_set_psf_scale(self.h, sx, sy)

    def set_finesampling(self, fs: int):
        self._check(self.lib.pfo_set_finesampling(self.h, fs))

    def set_return_finesampled(self, v: bool):
        self.lib.pfo_set_return_finesampled(self.h, int(v))

    def set_convolver(self, kind: str = "brute", omp_threads: int = 1):
        self._check(self.lib.pfo_set_convolver(self.h, kind.encode()))

    def set_omp_threads(self, n: int):
        self.lib.pfo_set_threads(self.h, n)

    def drawing_dims(self) -> Tuple[int, int]:
        w, h = C.c_uint(), C.c_uint()
        self._check(self.lib.pfo_drawing_dims(self.h, C.byref(w), C.byref(h)))
        return w.value, h.value

    def evaluate(self) -> Tuple[np.ndarray, Tuple[int, int]]:
        dw, dh = self.drawing_dims()
        cap = max(dw * dh, 1)
        buf = np.zeros(cap, dtype=np.float64)
        w, h, ox, oy = C.c_uint(), C.c_uint(), C.c_int(), C.c_int()
        self._check(self.lib.pfo_evaluate(self.h, buf.ctypes.data_as(_dp), cap, C.byref(w),
                                          C.byref(h), C.byref(ox), C.byref(oy)))
        return buf[: w.value * h.value].reshape(h.value, w.value).copy(), (ox.value, oy.value)

    def decisions(self, idx: int) -> np.ndarray:
        dw, dh = self.drawing_dims()
        out = np.zeros(dw * dh, dtype=np.int32)
        self._check(self.lib.pfo_decisions(self.h, idx, out.ctypes.data_as(C.POINTER(C.c_int)), out.size))
        return out.reshape(dh, dw)

    def level_counts(self, idx: int, max_levels: int = 16) -> list:
        out = (C.c_long * max_levels)()
        n = self.lib.pfo_level_counts(self.h, idx, out, max_levels)
        self._check(n)
        return [out[i] for i in range(n)]

    def evaluations(self, idx: int) -> int:
        """evaluate_at calls of the last evaluation of profile idx."""
        n = self.lib.pfo_evaluations(self.h, idx)
        self._check(n)
        return int(n)

    def scalars(self, idx: int) -> Dict[str, float]:
        out = np.zeros(len(SCALAR_NAMES))
        self._check(self.lib.pfo_profile_scalars(self.h, idx, out.ctypes.data_as(_dp), out.size))
        return dict(zip(SCALAR_NAMES, out.tolist()))


def loglike_norm(image: np.ndarray, sigma: np.ndarray, model: np.ndarray,
                 region: Optional[np.ndarray] = None) -> float:
    """ProFit's "norm" log-likelihood, R/profitLikeModel.R:263-276 (oracle restatement)."""
    lib = _OracleLib.get()
    im = np.ascontiguousarray(image, dtype=np.float64).ravel()
    sg = np.ascontiguousarray(sigma, dtype=np.float64).ravel()
    md = np.ascontiguousarray(model, dtype=np.float64).ravel()
    rg = None
    if region is not None:
        r = np.ascontiguousarray(region, dtype=np.uint8).ravel()
        rg = r.ctypes.data_as(C.POINTER(C.c_uint8))
    return lib.pfo_loglike_norm(im.ctypes.data_as(_dp), sg.ctypes.data_as(_dp),
                                md.ctypes.data_as(_dp), rg, im.size)


def loglike_other(kind: str, image: np.ndarray, sigma: np.ndarray, model: np.ndarray,
                  region: Optional[np.ndarray] = None) -> float:
    """profitLikeModel's chisq, t and pois log-likelihoods (oracle restatement,
    R/profitLikeModel.R:263-287 and 321-327), in FP64 with compensated sums:
      chisq: log dchisq(sum x^2, n), x = (image - model)/sigma over the region;
      t:     sum log dt(x, nu), nu = max(1, 2 v/(v - 1)), v = var(x) (n - 1 denominator);
      pois:  -sum(m - d log m) after scaling model and image by
             s = max(|image|/sigma^2) when s lies outside [0.1, 10]."""
    import math
    im = np.asarray(image, dtype=np.float64).ravel()
    sg = np.asarray(sigma, dtype=np.float64).ravel()
    md = np.asarray(model, dtype=np.float64).ravel()
    if region is not None:
        keep = np.asarray(region).ravel().astype(bool)
        im, sg, md = im[keep], sg[keep], md[keep]
    if kind == "pois":
        s = float(np.max(np.abs(im) / np.abs(sg) ** 2))
        if s < 0.1 or s > 10:
            md, im = md * s, im * s
        return -math.fsum(md - im * np.log(md))
    x = (im - md) / sg
    n = x.size
    if kind == "chisq":
        X2 = math.fsum(x * x)
        return (n / 2 - 1) * math.log(X2) - X2 / 2 - (n / 2) * math.log(2.0) - math.lgamma(n / 2)
    if kind == "t":
        mean = math.fsum(x) / n
        v = math.fsum((x - mean) ** 2) / (n - 1)
        nu = math.inf if v == 1 else max(1.0, 2 * v / (v - 1))
        if math.isinf(nu):
            return math.fsum(-(0.5 * math.log(2 * math.pi) + 0.5 * x * x))
        c0 = math.lgamma((nu + 1) / 2) - math.lgamma(nu / 2) - 0.5 * math.log(nu * math.pi)
        return n * c0 + math.fsum(-0.5 * (nu + 1) * np.log1p(x * x / nu))
    raise ValueError(kind)
