"""The gradient oracle: FP64 central finite differences of the compiled
reference, with a decision-log check at +-h.

libprofit has no gradient, so the oracle for d logL / d theta is a central
difference of the reference's own model (libprofit compiled in place,
``oracle/_ref``) and the "norm" likelihood of R/profitLikeModel.R:263-276
(restated with compensated sums in ``oracle/profit_oracle.c``).

The adjoint differentiates the chosen quadrature with every subsampling
decision held fixed.  A central difference is only comparable where nothing
piecewise-constant moves between theta - h and theta + h:
  * the subsampling decision of every pixel (radial.cpp:93-97, 326), and the
    resolution / rscale_max derived from re (radial.cpp:169-172): compared
    pixel by pixel through the restatement's decision log and its count of
    evaluate_at calls (which moves with the resolution);
  * the reference's own PROFIT_DEBUG counters of subsample_pixel calls per
    recursion level (radial.cpp:70-78).
A step at which either log differs from the one at theta is marked as
flipped and is not used for that component.

Test infrastructure only (imports the oracle).
"""
from __future__ import annotations

import os
from typing import Dict, List, Sequence, Tuple

import numpy as np

from oracle.pyoracle import OracleModel, RefModel, loglike_norm

RADIAL = {"sersic", "moffat", "ferrer", "ferrers", "coresersic", "king", "brokenexp"}


def _threads() -> int:
    return max(1, os.cpu_count() or 1)


def _with(profiles, overrides: Dict[int, Dict[str, float]]):
    out = []
    for i, (name, p) in enumerate(profiles):
        q = dict(p)
        q.update(overrides.get(i, {}))
        out.append((name, q))
    return out


def ref_loglike(wl: Dict, profiles, image: np.ndarray, sigma: np.ndarray, threads: int = 0) -> float:
    """logL of the compiled reference's model image (brute-force convolver,
    OpenMP threads) for the workload's geometry with `profiles`."""
    threads = threads or _threads()
    m = RefModel(wl["width"], wl["height"])
    m.set_magzero(wl["magzero"])
    if wl.get("psf") is not None:
        m.set_psf(wl["psf"])
    m.set_omp_threads(threads)
    m.set_convolver("brute", threads)
    for name, p in profiles:
        m.add_profile(name, **p)
    img, _ = m.evaluate()
    return loglike_norm(image, sigma, img)


def _decision_log(wl: Dict, profiles, only: int = -1) -> List[Tuple]:
    """Per radial profile: (per-pixel decisions, evaluate_at count) of the
    restatement and the PROFIT_DEBUG per-level counts of the reference.
    Profiles are drawn unconvolved: decisions do not depend on the PSF.  A
    profile's decisions depend on its own parameters only, so `only` >= 0
    draws just that profile."""
    if only >= 0:
        profiles = [profiles[only]]
    flat = [(n, {**p, "convolve": False} if n in RADIAL else p) for n, p in profiles]
    ora = OracleModel(wl["width"], wl["height"], threads=_threads())
    ora.set_magzero(wl["magzero"])
    dbg = RefModel(wl["width"], wl["height"], debug=True)
    dbg.set_magzero(wl["magzero"])
    dbg.set_omp_threads(1)
    for name, p in flat:
        ora.add_profile(name, **p)
        dbg.add_profile(name, **p)
    ora.evaluate()
    dbg.evaluate()
    log = []
    for i, (name, _) in enumerate(flat):
        if name in RADIAL:
            log.append((ora.decisions(i), ora.evaluations(i), tuple(dbg.integrations(i))))
    return log


def _same_log(a, b) -> bool:
    return all(np.array_equal(x[0], y[0]) and x[1] == y[1] and x[2] == y[2] for x, y in zip(a, b))


def ref_fd_gradient(wl: Dict, profiles, image: np.ndarray, sigma: np.ndarray,
                    refs: Sequence[Tuple[int, str]], rel_steps: Sequence[float] = (1e-7, 1e-6),
                    check_decisions: bool = True) -> Dict:
    """Central differences of the compiled reference's logL for every
    (profile index, parameter) of refs at each relative step
    (h = step * max(|theta|, 1)).

    Returns {"loglike": logL at theta, "grad": {step: array},
             "flipped": {step: bool array}} where flipped[step][k] says that
    a decision log at theta +- h differs from the one at theta."""
    ll0 = ref_loglike(wl, profiles, image, sigma)
    base = {}
    grads, flips = {}, {}
    for s in rel_steps:
        g = np.zeros(len(refs))
        f = np.zeros(len(refs), dtype=bool)
        for j, (pi, k) in enumerate(refs):
            v = profiles[pi][1][k]
            h = s * max(abs(v), 1.0)
            up = _with(profiles, {pi: {k: v + h}})
            dn = _with(profiles, {pi: {k: v - h}})
            g[j] = (ref_loglike(wl, up, image, sigma) - ref_loglike(wl, dn, image, sigma)) / (2 * h)
            if check_decisions and profiles[pi][0] in RADIAL:
                if pi not in base:
                    base[pi] = _decision_log(wl, profiles, pi)
                f[j] = not (_same_log(_decision_log(wl, up, pi), base[pi]) and
                            _same_log(_decision_log(wl, dn, pi), base[pi]))
        grads[s], flips[s] = g, f
    return {"loglike": ll0, "grad": grads, "flipped": flips}


def closest_error(g_ad: np.ndarray, fd: Dict) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Per component, the FD step (among those without a decision flip) that
    agrees best with the adjoint: returns (abs error, the FD value used,
    usable) where usable is False for components whose every step flipped."""
    steps = sorted(fd["grad"])
    best_err = np.full(len(g_ad), np.inf)
    best_ref = np.zeros(len(g_ad))
    for s in steps:
        ok = ~fd["flipped"][s]
        e = np.abs(g_ad - fd["grad"][s])
        take = ok & (e < best_err)
        best_err[take] = e[take]
        best_ref[take] = fd["grad"][s][take]
    usable = np.isfinite(best_err)
    return best_err, best_ref, usable


def gradient_errors(g_ad: np.ndarray, fd: Dict) -> Dict:
    """The errors the FP32 bar is stated in, over the components with a
    flip-free FD step:
      own:  |g_ad - g_ref| / |g_ref| per component,
      norm: ||g_ad - g_ref|| / ||g_ref|| (the vector's relative error),
      of_norm: |g_ad - g_ref| / ||g_ref|| per component."""
    err, ref, usable = closest_error(g_ad, fd)
    e, r = err[usable], ref[usable]
    nrm = float(np.linalg.norm(r))
    return {"own": e / np.maximum(np.abs(r), 1e-300), "norm": float(np.linalg.norm(e)) / nrm, "of_norm": e / nrm,
            "usable": usable, "ref": ref}
