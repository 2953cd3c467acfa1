"""Fit-space transforms and priors (profit_b200.fit) on the host: the remake
follows profitRemakeModellist's rules, and d LP / d parm matches central
differences of LP for a smooth stand-in likelihood (logged, clamped and tied
parameters, normal and flat priors)."""
import math

import numpy as np
import pytest

from profit_b200.fit import FitSpace

# (1, "nser") is tied to (0, "nser") just before it, like ProFit's
# nser = c(2.5, NA) unlisted as nser1, nser2
PARAMS = [(0, "xcen"), (0, "ycen"), (0, "mag"), (0, "re"), (0, "nser"), (1, "nser"), (1, "axrat")]
INIT = [50.0, 48.0, 17.0, 6.0, 2.5, 2.5, 0.6]


def _quadratic_ll(params, theta):
    """A smooth likelihood in model space with a known gradient."""
    c = np.array([51.0, 47.5, 17.3, 7.0, 2.2, 5.0, 0.7])
    w = np.array([0.5, 0.8, 3.0, 0.2, 1.5, 0.3, 4.0])
    d = np.asarray(theta) - c
    return float(-np.sum(w * d * d)), -2 * w * d


def _space():
    return FitSpace(PARAMS, INIT, tofit=[True, True, True, True, True, None, True],
                    tolog=[False, False, False, True, True, True, False],
                    intervals=[None, None, (10, 30), (0.5, 100), (0.5, 3.0), None, (0.05, 1.0)],
                    prior_sigmas=[2.0, 2.0, math.inf, 0.3, 0.2, 0.3, 0.5])


def test_remake_follows_profit_rules():
    fs = _space()
    parm = fs.initial_parm()
    assert np.allclose(parm, [50, 48, 17, math.log10(6), math.log10(2.5), 0.6])
    theta, _, out = fs.remake(parm)
    assert np.allclose(theta, INIT)
    assert theta[5] == theta[4]  # tied to the parameter before it
    # clamping: nser beyond its interval comes back at the edge, in fit space
    p2 = parm.copy()
    p2[4] = math.log10(5.0)
    theta2, deriv2, out2 = fs.remake(p2)
    assert theta2[4] == 3.0 and deriv2[4] == 0.0 and out2[4] == pytest.approx(math.log10(3.0))
    assert theta2[5] == 3.0  # re-inherited after the clamp
    with pytest.raises(ValueError):
        fs.remake(parm[:-1])


@pytest.mark.parametrize("shift", [0.0, 0.05])
def test_lp_gradient_matches_finite_differences(shift):
    fs = _space()
    parm = fs.initial_parm() + shift
    lp, g, _ = fs.lp_grad(parm, _quadratic_ll)
    h = 1e-6
    fd = np.zeros_like(g)
    for j in range(len(parm)):
        pp, pm = parm.copy(), parm.copy()
        pp[j] += h
        pm[j] -= h
        fd[j] = (fs.lp_grad(pp, _quadratic_ll)[0] - fs.lp_grad(pm, _quadratic_ll)[0]) / (2 * h)
    np.testing.assert_allclose(g, fd, rtol=1e-6, atol=1e-6)


def test_prior_matches_profit_make_priors_form():
    fs = _space()
    theta = np.array(INIT)
    theta[0] += 1.0
    lp, _ = fs.log_prior(theta)
    # normal on xcen (sigma 2) and ycen, on log10 for re/nser, flat for mag, axrat normal
    want = 0.0
    for i, s in enumerate([2.0, 2.0, math.inf, 0.3, 0.2, 0.3, 0.5]):
        if i == 5 or not math.isfinite(s):
            continue  # tied (not fitted) or flat
        x, mu = theta[i], INIT[i]
        if i in (3, 4):
            x, mu = math.log10(x), math.log10(mu)
        want += -0.5 * math.log(2 * math.pi) - math.log(s) - 0.5 * ((x - mu) / s) ** 2
    assert lp == pytest.approx(want, rel=1e-14)


@pytest.mark.gpu
def test_lp_gradient_with_the_device_adjoint():
    """LP and d LP / d parm with the FP32 adjoint likelihood gradient, against
    central differences of LP built on the plain FP64 likelihood."""
    from profit_b200 import PF_FP32, PF_FP64, Model
    from profit_b200 import workloads as W
    from profit_b200.fit import model_loglike_grad
    wl = W.single_sersic(seed_tag=21, width=90, height=80, psf_size=15)
    m = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m.evaluate()
    image, sigma = W.make_data(wl, truth)
    m.set_data(image, sigma)
    refs = wl["grad"][:7]  # xcen ycen mag re nser ang axrat
    init = [wl["profiles"][0][1][k] for (_, k) in refs]
    fs = FitSpace(refs, init, tofit=[True] * 7, tolog=[False, False, False, True, True, False, True],
                  intervals=[None, None, None, (0.5, 50), (0.5, 8), None, (0.05, 1)],
                  prior_sigmas=[1.0, 1.0, math.inf, 0.2, 0.2, 30.0, 0.3])
    parm = fs.initial_parm() + np.array([0.3, -0.2, 0.05, 0.02, -0.02, 2.0, 0.01])
    m.set_precision(PF_FP32)
    lp, g, _ = fs.lp_grad(parm, model_loglike_grad(m))
    m.set_precision(PF_FP64)

    def lp64(p):
        theta, _, _ = fs.remake(p)
        m.set_parameters(refs, theta)
        return m.loglike() + fs.log_prior(theta)[0]

    assert lp == pytest.approx(lp64(parm), rel=1e-6)
    fd = np.zeros(len(parm))
    for j in range(len(parm)):
        h = 1e-6 * max(abs(parm[j]), 1.0)
        pp, pm = parm.copy(), parm.copy()
        pp[j] += h
        pm[j] -= h
        fd[j] = (lp64(pp) - lp64(pm)) / (2 * h)
    np.testing.assert_allclose(g, fd, rtol=1e-4, atol=1e-5 * np.max(np.abs(fd)))
