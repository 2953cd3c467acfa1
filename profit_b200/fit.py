"""Fit-space parameters and priors around the likelihood, as ProFit's R layer
has them: profitRemakeModellist (R/profitRemakeModelList.R:27-166) maps the
sampler's parameter vector to model parameters (tofit, tolog, offsets, ties,
interval clamps), profitMakePriors (R/profitUtility.R:124-176) builds normal
priors, and profitLikeModel returns LP = LL + priors (R/profitLikeModel.R:
225-240, 342).

On top of ProFit this gives d LP / d parm in fit space: the device adjoint
gradient d LL / d theta (theta the model parameters) chained through the
transforms.

    value_i = 10^parm_i if tolog_i else parm_i      (fitted entries; init otherwise)
    value_i = (value_i + offset shift) * offset size   (by parameter name)
    theta_i = clamp(value_i, interval_i), or theta_{i-1} for a tied entry
    d theta_i / d parm_i = (0 if clamped else 1) * (theta_i ln 10 if tolog_i else 1)
                           * (offset size for size parameters)

A parameter whose tofit entry is None takes the value of the one before it
(ProFit's NA), after the clamps, and its gradient flows to that parameter.
Priors are normal on theta, or on log10(theta) where the prior's tolog is set,
evaluated at the clamped values, on every entry (profitMakePriors without
tofit) or on those prior_on selects; an infinite sigma means a flat prior
(profitMakePriors' allowflat).

FitSpace is the host form of the mapping (one proposal at a time, any
likelihood callable).  FitSpace.install(model) puts the same mapping on a
profit_b200.Model, whose lp_grad_batch(parm) then evaluates LP and
d LP / d parm for whole batches with the mapping on the device.
"""
from __future__ import annotations

import math
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

LN10 = math.log(10.0)


class FitSpace:
    """params: (profile index, name) of every model parameter in the mapping,
    in ProFit's unlist(modellist) order for ties; init: their model-space
    values; tofit: True (fitted), False (fixed at init) or None (tied to the
    parameter before it); tolog: fit log10 of the value; intervals: (lo, hi)
    or None per parameter (model space); prior_sigmas / prior_means /
    prior_tolog: profitMakePriors' arguments (None: no priors; means default
    to init)."""

    def __init__(self, params: Sequence[Tuple[int, str]], init: Sequence[float],
                 tofit: Sequence[Optional[bool]], tolog: Optional[Sequence[bool]] = None,
                 intervals: Optional[Sequence[Optional[Tuple[float, float]]]] = None,
                 prior_sigmas: Optional[Sequence[float]] = None, prior_means: Optional[Sequence[float]] = None,
                 prior_tolog: Optional[Sequence[bool]] = None, offset: Optional[Sequence[float]] = None,
                 prior_on: Optional[Sequence[bool]] = None, names: Optional[Sequence[str]] = None):
        n = len(params)
        self.params = list(params)
        self.init = np.asarray(init, dtype=np.float64)
        self.tofit = list(tofit)
        self.tolog = np.zeros(n, bool) if tolog is None else np.asarray(tolog, dtype=bool)
        self.intervals = [None] * n if intervals is None else list(intervals)
        if not (len(self.init) == len(self.tofit) == len(self.tolog) == len(self.intervals) == n):
            raise ValueError("params, init, tofit, tolog and intervals must have the same length")
        if n and self.tofit[0] is None:
            raise ValueError("the first parameter cannot inherit (tofit None) from a previous one")
        self.fit_ids = [i for i, f in enumerate(self.tofit) if f is True]
        self.sigmas = None if prior_sigmas is None else np.asarray(prior_sigmas, dtype=np.float64)
        self.means = self.init.copy() if prior_means is None else np.asarray(prior_means, dtype=np.float64)
        self.prior_tolog = self.tolog.copy() if prior_tolog is None else np.asarray(prior_tolog, dtype=bool)
        if self.sigmas is not None and (len(self.sigmas) != n or np.any(self.sigmas <= 0)):
            raise ValueError("prior sigmas must be positive, one per parameter")
        self.prior_on = np.ones(n, bool) if prior_on is None else np.asarray(prior_on, dtype=bool)
        # R's offset: xcen/ycen/ang shifts, then size parameters scaled
        self.offset = None if offset is None else [float(v) for v in offset]
        names = [nm for (_, nm) in self.params] if names is None else list(names)
        self._shift = np.zeros(n)
        self._scale = np.ones(n)
        if self.offset is not None:
            ox, oy, oang, osize = self.offset
            for i, nm in enumerate(names):
                if nm == "xcen":
                    self._shift[i] = ox
                elif nm == "ycen":
                    self._shift[i] = oy
                elif nm == "ang" and not math.isnan(oang):
                    self._shift[i] = oang
                if nm in ("xcen", "ycen", "re", "fwhm", "rb", "rout", "rc", "rt") and not math.isnan(osize):
                    self._scale[i] = osize

    def initial_parm(self) -> np.ndarray:
        """The sampler's starting vector (profitSetupData's init in fit space)."""
        v = self.init[self.fit_ids]
        return np.where(self.tolog[self.fit_ids], np.log10(v), v)

    def remake(self, parm: Sequence[float]) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
        """profitRemakeModellist: (theta, dtheta/dparm for the fitted entries,
        the clamped parm to hand back to the sampler)."""
        parm = np.asarray(parm, dtype=np.float64)
        if parm.shape[-1] != len(self.fit_ids):
            raise ValueError("length of parm mismatches the number of fitted parameters")
        theta = self.init.copy()
        deriv = np.ones(len(theta))
        for j, i in enumerate(self.fit_ids):
            if self.tolog[i]:
                theta[i] = 10.0 ** parm[j]
                deriv[i] = theta[i] * LN10
            else:
                theta[i] = parm[j]
        theta = (theta + self._shift) * self._scale
        deriv = deriv * self._scale
        for i, f in enumerate(self.tofit):
            if f is None:
                theta[i] = theta[i - 1]
        for i, iv in enumerate(self.intervals):
            if iv is None:
                continue
            lo, hi = iv
            v = max(lo, min(hi, theta[i]))
            if v != theta[i]:
                deriv[i] = 0.0  # clamped: the value no longer moves with parm
            theta[i] = v
        for i, f in enumerate(self.tofit):  # re-inherit after the clamps
            if f is None:
                theta[i] = theta[i - 1]
        out = (theta[self.fit_ids] - self._shift[self.fit_ids]) / self._scale[self.fit_ids]
        out = np.where(self.tolog[self.fit_ids], np.log10(out), out)
        return theta, deriv, out

    def log_prior(self, theta: np.ndarray) -> Tuple[float, np.ndarray]:
        """profitMakePriors' normal priors at theta and their derivative in theta."""
        g = np.zeros(len(theta))
        if self.sigmas is None:
            return 0.0, g
        lp = 0.0
        for i in np.flatnonzero(self.prior_on):
            s = self.sigmas[i]
            if not math.isfinite(s):
                continue  # flat
            if self.prior_tolog[i]:
                x, mu = math.log10(theta[i]), math.log10(self.means[i])
                lp += -0.5 * math.log(2 * math.pi) - math.log(s) - 0.5 * ((x - mu) / s) ** 2
                g[i] = -(x - mu) / (s * s) / (theta[i] * LN10)
            else:
                x, mu = theta[i], self.means[i]
                lp += -0.5 * math.log(2 * math.pi) - math.log(s) - 0.5 * ((x - mu) / s) ** 2
                g[i] = -(x - mu) / (s * s)
        return lp, g

    def chain(self, dtheta: np.ndarray, deriv: np.ndarray) -> np.ndarray:
        """d/dparm from d/dtheta: ties flow to their source, then the
        transform and clamp factors of the fitted entries."""
        d = np.array(dtheta, dtype=np.float64)
        for i in reversed(range(len(self.tofit))):
            if self.tofit[i] is None:
                d[i - 1] += d[i]
                d[i] = 0.0
        return np.array([d[i] * deriv[i] for i in self.fit_ids])

    def install(self, model) -> None:
        """Puts this mapping on a profit_b200.Model (pf_model_set_fit_space):
        model.lp_grad_batch(parm) then evaluates LP, d LP / d parm, the
        returned parm and LL for a batch of fitted vectors on the device."""
        model.set_fit_space(self.params, self.init, self.tofit, self.tolog, self.intervals, self.offset,
                            None if self.sigmas is None else self.sigmas, self.means, self.prior_tolog,
                            self.prior_on)

    def lp_grad(self, parm: Sequence[float],
                loglike_grad: Callable[[Sequence[Tuple[int, str]], np.ndarray], Tuple[float, np.ndarray]]
                ) -> Tuple[float, np.ndarray, np.ndarray]:
        """LP = LL + priors at parm, d LP / d parm, and the clamped parm.
        loglike_grad(params, theta) returns (LL, d LL / d theta), e.g.
        model_loglike_grad(model)."""
        theta, deriv, parm_out = self.remake(parm)
        ll, g_ll = loglike_grad(self.params, theta)
        lp_prior, g_prior = self.log_prior(theta)
        return ll + lp_prior, self.chain(np.asarray(g_ll) + g_prior, deriv), parm_out


def model_loglike_grad(model) -> Callable:
    """LL and its adjoint gradient from a profit_b200.Model (FP32 path)."""
    def f(params, theta):
        model.set_parameters(params, theta)
        return model.loglike_grad(params)
    return f
