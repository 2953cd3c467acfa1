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


TOFIT = [True, True, True, True, True, None, True]


def _space(**kw):
    return FitSpace(PARAMS, INIT, tofit=TOFIT,
                    tolog=[False, False, False, True, True, True, False],
                    intervals=[None, None, (10, 30), (0.5, 100), (0.5, 3.0), None, (0.05, 1.0)],
                    prior_sigmas=[2.0, 2.0, math.inf, 0.3, 0.2, 0.3, 0.5], **kw)


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


@pytest.mark.parametrize("with_tofit", [True, False])
def test_prior_matches_profit_make_priors_form(with_tofit):
    """profitMakePriors(modellist, sigmas, tolog, tofit = tofit) puts priors on
    the fitted entries only; without tofit (its default) on every entry."""
    fs = _space(prior_on=[f is True for f in TOFIT] if with_tofit else None)
    theta = np.array(INIT)
    theta[0] += 1.0
    lp, _ = fs.log_prior(theta)
    # normal on xcen (sigma 2) and ycen, on log10 for re/nser, flat for mag, axrat normal
    want = 0.0
    for i, s in enumerate([2.0, 2.0, math.inf, 0.3, 0.2, 0.3, 0.5]):
        if (with_tofit and i == 5) or not math.isfinite(s):
            continue  # tied (not fitted) or flat
        x, mu = theta[i], INIT[i]
        if i in (3, 4, 5):
            x, mu = math.log10(x), math.log10(mu)
        want += -0.5 * math.log(2 * math.pi) - math.log(s) - 0.5 * ((x - mu) / s) ** 2
    assert lp == pytest.approx(want, rel=1e-14)


def test_offsets_follow_profit_remake_modellist():
    """R's offset: xcen/ycen/ang shifted, then xcen, ycen and sizes scaled;
    the returned parm takes the shifts off before the scale."""
    params = [(0, "xcen"), (0, "ycen"), (0, "re"), (0, "ang"), (0, "mag")]
    init = [50.0, 40.0, 6.0, 30.0, 17.0]
    fs = FitSpace(params, init, tofit=[True] * 5, tolog=[False, False, True, False, False],
                  offset=[1.5, -2.0, 10.0, 2.0])
    parm = fs.initial_parm()
    theta, deriv, out = fs.remake(parm)
    assert np.allclose(theta, [(50 + 1.5) * 2, (40 - 2.0) * 2, 6.0 * 2, 40.0, 17.0])
    assert np.allclose(deriv, [2.0, 2.0, 12.0 * math.log(10), 1.0, 1.0])
    assert np.allclose(out, [(103.0 - 1.5) / 2, (76.0 + 2.0) / 2, math.log10(6.0), 30.0, 17.0])


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


def _two_sersic_space():
    """Bulge + disk in unlist(modellist) order (xcen1, xcen2, ycen1, ...):
    the disk's centre tied to the bulge's (R's NA), sizes and indices fitted
    in log10, the disk's nser and both boxes fixed, an interval on each axis
    ratio, an offset, and priors (flat on the magnitudes)."""
    from profit_b200 import workloads as W
    wl = W.bulge_disk_ps(width=120, height=110, psf_size=15)
    wl["profiles"] = wl["profiles"][:2]
    b, d = wl["profiles"][0][1], wl["profiles"][1][1]
    names = ["xcen", "ycen", "mag", "re", "nser", "ang", "axrat", "box"]
    params, init, tofit, tolog, iv, sig = [], [], [], [], [], []
    for k in names:
        for pi, p in ((0, b), (1, d)):
            params.append((pi, k))
            init.append(p[k])
            tied = pi == 1 and k in ("xcen", "ycen")
            fixed = k == "box" or (pi == 1 and k == "nser")
            tofit.append(None if tied else (False if fixed else True))
            tolog.append(k in ("re", "nser"))
            iv.append((0.1, 1.0) if k == "axrat" else ((0.5, 10.0) if k == "nser" else None))
            sig.append(math.inf if k == "mag" else {"xcen": 2.0, "ycen": 2.0, "re": 0.3, "nser": 0.3, "ang": 20.0,
                                                    "axrat": 0.3, "box": 0.1}[k])
    fs = FitSpace(params, init, tofit, tolog=tolog, intervals=iv, prior_sigmas=sig, offset=[0.4, -0.3, 2.0, 1.01])
    return wl, fs


@pytest.mark.gpu
@pytest.mark.parametrize("batch", [4, 40])
def test_device_fit_space_matches_host_restatement(batch):
    """pf_model_lp_grad_batch (the mapping and chain rule on the device for
    40 proposals, on the host for 4) against FitSpace.lp_grad around the
    model's FP32 adjoint, row by row; a proposal whose axis ratio leaves its
    interval comes back clamped with a zero gradient in that entry."""
    from profit_b200 import PF_FP32, Model
    from profit_b200 import workloads as W
    from profit_b200.fit import model_loglike_grad
    wl, fs = _two_sersic_space()
    m64 = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m64.evaluate()
    image, sigma = W.make_data(wl, truth)
    r = np.random.Generator(np.random.PCG64(44))
    p0 = fs.initial_parm()
    parm = p0 + r.normal(size=(batch, len(p0))) * 0.01 * np.maximum(np.abs(p0), 0.1)
    ax = [j for j, i in enumerate(fs.fit_ids) if fs.params[i][1] == "axrat"][0]
    parm[1, ax] = 1.2  # beyond the interval: clamped to 1
    dev = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    dev.set_data(image, sigma)
    fs.install(dev)
    assert dev.fit_size() == (len(fs.fit_ids), len(fs.params))
    lp, g, pout, ll = dev.lp_grad_batch(parm)
    host = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    host.set_data(image, sigma)
    for b in range(batch):
        lp_h, g_h, out_h = fs.lp_grad(parm[b], model_loglike_grad(host))
        # two FP32 renders add their subsampled cells to the pixels in
        # different (atomic) orders: at this brightness logL moves by ~1e-7
        assert lp[b] == pytest.approx(lp_h, rel=1e-6)
        np.testing.assert_allclose(pout[b], out_h, rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(g[b], g_h, rtol=1e-5, atol=1e-6 * np.max(np.abs(g_h)))
    assert pout[1, ax] == pytest.approx(1.0) and g[1, ax] == 0.0
    theta, _, _ = fs.remake(parm[0])
    assert lp[0] - ll[0] == pytest.approx(fs.log_prior(theta)[0], rel=1e-12)


@pytest.mark.gpu
def test_device_fit_space_gradient_matches_fd64():
    """d LP / d parm from the device fit space against central differences of
    LP formed with the plain FP64 likelihood."""
    from profit_b200 import PF_FP32, PF_FP64, Model
    from profit_b200 import workloads as W
    wl, fs = _two_sersic_space()
    m64 = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m64.evaluate()
    image, sigma = W.make_data(wl, truth)
    p0 = fs.initial_parm()
    parm = p0 + np.linspace(-0.01, 0.01, len(p0)) * np.maximum(np.abs(p0), 0.1)
    dev = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    dev.set_data(image, sigma)
    fs.install(dev)
    lp, g, _, _ = dev.lp_grad_batch(parm[None, :])
    m64.set_data(image, sigma)
    m64.set_precision(PF_FP64)
    theta_refs = fs.params

    def lp64(p):
        theta, _, _ = fs.remake(p)
        m64.set_parameters(theta_refs, theta)
        return m64.loglike() + fs.log_prior(theta)[0]

    assert lp[0] == pytest.approx(lp64(parm), rel=1e-6)
    fd6, fd5 = np.zeros(len(parm)), np.zeros(len(parm))
    for fd, step in ((fd6, 1e-6), (fd5, 1e-5)):
        for j in range(len(parm)):
            h = step * max(abs(parm[j]), 1.0)
            pp, pm = parm.copy(), parm.copy()
            pp[j] += h
            pm[j] -= h
            fd[j] = (lp64(pp) - lp64(pm)) / (2 * h)
    scale = np.max(np.abs(fd6))
    err = np.minimum(np.abs(g[0] - fd6), np.abs(g[0] - fd5)) / scale
    assert np.all(err <= 1e-5), list(zip(fs.fit_ids, fd6, fd5, g[0]))
