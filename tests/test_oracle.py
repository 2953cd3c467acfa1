"""Pins the oracle (CPU, no GPU needed).

1. The R-math / QUADPACK stand-ins used to compile libprofit agree with
   scipy (scipy.integrate.quad wraps the Fortran QUADPACK that R's
   Rdqags/Rdqagi translate, so results match to the last bits).
2. The plain-C restatement (oracle/profit_oracle.c) reproduces the compiled
   reference bit for bit on rendering, and to rounding with convolution.
3. Decision counters of the restatement equal libprofit's PROFIT_DEBUG
   counters (radial.cpp:70-78).
4. The likelihood restatement equals sum(log N(x; 0, 1)) (R's dnorm).
"""
import math

import numpy as np
import pytest
from scipy import integrate, special, stats

from oracle.pyoracle import OracleModel, RefModel, loglike_norm, ref_integrate, ref_special
from profit_b200 import workloads as W

# (profile, params) exercising every radial profile, boxy and rotated shapes
# and Sersic's pow-avoiding specialisations (sersic.cpp:225-252).
PROFILE_CASES = [
    ("sersic", dict(xcen=50.3, ycen=49.7, mag=15, re=8, nser=2.5, ang=30, axrat=0.6)),
    ("sersic", dict(xcen=47.1, ycen=52.2, mag=15, re=5.5, nser=4, ang=120, axrat=0.45, box=0.2)),
    ("sersic", dict(xcen=50.0, ycen=50.0, mag=15, re=1.5, nser=0.5, ang=10, axrat=0.9)),
    ("sersic", dict(xcen=50.5, ycen=50.5, mag=15, re=3, nser=8, ang=10, axrat=0.9)),
    ("sersic", dict(xcen=40.2, ycen=61.3, mag=14, re=20, nser=1, ang=75, axrat=0.3)),
    ("sersic", dict(xcen=50.1, ycen=50.2, mag=15, re=6, nser=2, ang=5, axrat=0.8, box=-0.3)),
    ("sersic", dict(xcen=50.1, ycen=50.2, mag=15, re=6, nser=3, ang=5, axrat=0.8)),
    ("moffat", dict(xcen=50.2, ycen=50.6, mag=16, fwhm=3, con=2.5, ang=40, axrat=0.7)),
    ("moffat", dict(xcen=48.2, ycen=51.6, mag=16, fwhm=6, con=1.5, ang=100, axrat=0.5, box=0.4)),
    ("ferrer", dict(xcen=50.2, ycen=49.6, mag=16, rout=20, a=1.5, b=0.5, ang=40, axrat=0.7)),
    ("coresersic", dict(xcen=50.2, ycen=49.6, mag=16, re=10, rb=2, nser=3, a=2, b=0.5, ang=40, axrat=0.7)),
    ("king", dict(xcen=50.2, ycen=49.6, mag=16, rc=3, rt=30, a=2, ang=70, axrat=0.8, box=-0.2)),
    ("brokenexp", dict(xcen=50.2, ycen=49.6, mag=16, h1=6, h2=3, rb=12, a=1, ang=70, axrat=0.8)),
]


@pytest.mark.parametrize("a", [1.0, 2.0, 3.5, 5.0, 8.0, 16.0, 20.0])
@pytest.mark.parametrize("p", [0.5, 0.9999, 0.995, 0.1])
def test_qgamma_matches_scipy(a, p):
    q = ref_special()["qgamma"](p, a)
    assert q == pytest.approx(special.gammaincinv(a, p), rel=2e-15)


@pytest.mark.parametrize("a", [0.3, 1.0, 5.5, 20.0])
@pytest.mark.parametrize("x", [0.1, 1.0, 5.0, 30.0])
def test_pgamma_beta_gamma(a, x):
    sp = ref_special()
    assert sp["pgamma"](x, a) == pytest.approx(special.gammainc(a, x), rel=1e-14, abs=1e-300)
    assert sp["beta"](a, x) == pytest.approx(special.beta(a, x), rel=1e-13)
    assert sp["gammafn"](a) == pytest.approx(special.gamma(a), rel=1e-14)


def _king(r, rc=3.0, rt=30.0, a=2.0):
    if r >= rt:
        return 0.0
    return r * (1 / (1 + (r / rc) ** 2) ** (1 / a) - 1 / (1 + (rt / rc) ** 2) ** (1 / a)) ** a


def _brokenexp(r, h1=6.0, h2=3.0, rb=12.0, a=1.0):
    base = r - rb
    if a * base < 40:
        base = math.log(1 + math.exp(a * base)) / a
    return r * math.exp(-r / h1 + (1 / h1 - 1 / h2) * base)


def _coresersic(r, re=10.0, rb=2.0, nser=3.0, a=2.0, b=0.5):
    if r <= 0:
        return 0.0
    bn = special.gammaincinv(2 * nser, 0.5)
    return r * (1 + (r / rb) ** -a) ** (b / a) * math.exp(-bn * ((r ** a + rb ** a) / re ** a) ** (1 / (nser * a)))


def test_quadpack_matches_scipy_quad():
    # finite range (dqags) and semi-infinite (dqagi), libprofit's tolerances
    assert ref_integrate(_king, 0.0, 30.0) == integrate.quad(_king, 0, 30.0, epsabs=1e-4, epsrel=1e-4, limit=100)[0]
    for f in (_brokenexp, _coresersic):
        ours = ref_integrate(f, 0.0)
        theirs = integrate.quad(f, 0, np.inf, epsabs=1e-4, epsrel=1e-4, limit=100)[0]
        assert ours == pytest.approx(theirs, rel=1e-14)


@pytest.mark.parametrize("case", range(len(PROFILE_CASES)))
def test_restatement_bit_exact_render(case):
    name, params = PROFILE_CASES[case]
    ref = RefModel(100, 100)
    ref.add_profile(name, **params)
    a, _ = ref.evaluate()
    ora = OracleModel(100, 100)
    ora.add_profile(name, **params)
    b, _ = ora.evaluate()
    assert np.array_equal(a, b)
    # total flux 10^(-0.4 (mag - magzero)) when the profile fits the image (radial.cpp:149-152)
    compact = (name == "sersic" and params["re"] < 10 and params["nser"] <= 4) or \
              (name == "moffat" and params["con"] >= 2)
    if compact:
        assert a.sum() == pytest.approx(10 ** (-0.4 * params["mag"]), rel=0.05)


@pytest.mark.parametrize("wl", [W.single_sersic(), W.bulge_disk_ps(width=160, height=140, psf_size=25)],
                         ids=["single_sersic", "bulge_disk_ps_small"])
def test_restatement_with_convolution(wl):
    ref = W.configure(RefModel(wl["width"], wl["height"]), wl)
    a, off_a = ref.evaluate()
    ora = W.configure(OracleModel(wl["width"], wl["height"]), wl)
    b, off_b = ora.evaluate()
    assert a.shape == b.shape and off_a == off_b
    assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(a))


def test_restatement_sky_psf_point_source():
    psf = W.moffat_psf(15, 3.0, 2.5)
    out = []
    for M in (RefModel, OracleModel):
        m = M(60, 50)
        m.set_psf(psf)
        m.add_profile("sersic", xcen=30, ycen=25, re=4, nser=2, convolve=True)
        m.add_profile("sky", bg=0.25)
        m.add_profile("psf", xcen=12.3, ycen=40.6, mag=14)
        out.append(m.evaluate()[0])
    assert np.max(np.abs(out[0] - out[1])) <= 1e-13 * np.max(np.abs(out[0]))


@pytest.mark.parametrize("case", [0, 1, 3, 7, 9, 10])
def test_decision_counts_match_profit_debug(case):
    name, params = PROFILE_CASES[case]
    ref = RefModel(100, 100, debug=True)
    ref.set_omp_threads(1)
    ref.add_profile(name, **params)
    ref.evaluate()
    ora = OracleModel(100, 100)
    ora.add_profile(name, **params)
    ora.evaluate()
    assert ora.level_counts(0) == ref.integrations(0)
    d = ora.decisions(0)
    assert int(d[d > 0].sum()) == sum(ref.integrations(0))


@pytest.mark.parametrize("case", [7, 9, 11])
def test_evaluation_count_from_profit_debug(case):
    """The oracle's evaluate_at count: one per directly evaluated pixel, and
    res^2 sub-points per subsample_pixel call, each evaluated twice (value and
    test point) below max_recursions = 2 and once at the last level
    (radial.cpp:54-134).  Profiles without a centre override use one
    resolution for every cell, so the count follows from PROFIT_DEBUG's
    per-level counters of the compiled reference."""
    name, params = PROFILE_CASES[case]
    ref = RefModel(100, 100, debug=True)
    ref.set_omp_threads(1)
    ref.add_profile(name, **params)
    ref.evaluate()
    ora = OracleModel(100, 100)
    ora.add_profile(name, **params)
    ora.evaluate()
    res = int(ora.scalars(0)["resolution"])
    direct = int(np.sum(ora.decisions(0) == 0))
    sub_evals = sum(c * res * res * (2 if level < 2 else 1) for level, c in enumerate(ref.integrations(0)))
    assert ora.evaluations(0) == direct + sub_evals


def test_evaluation_count_rough():
    """rough = true evaluates each pixel inside rscale_max once."""
    name, params = PROFILE_CASES[0]
    ora = OracleModel(100, 100)
    ora.add_profile(name, rough=True, **params)
    ora.evaluate()
    assert ora.evaluations(0) == int(np.sum(ora.decisions(0) == 0))


def test_loglike_restatement():
    r = np.random.default_rng(5)
    model = r.uniform(0, 3, size=(40, 30))
    sigma = r.uniform(0.5, 2, size=model.shape)
    image = model + r.normal(size=model.shape) * sigma
    ll = loglike_norm(image, sigma, model)
    assert ll == pytest.approx(stats.norm.logpdf((image - model) / sigma).sum(), rel=1e-13)
    region = r.uniform(size=model.shape) > 0.3
    ll_r = loglike_norm(image, sigma, model, region)
    assert ll_r == pytest.approx(stats.norm.logpdf(((image - model) / sigma)[region]).sum(), rel=1e-13)


def test_fft_geometry_restatement_matches_numpy_fft():
    """The FFT convolver restatement equals libprofit's 1-D r2c over the
    flattened 2*max(src, krn) buffer (convolve.cpp:245-312, fft.cpp:113-158),
    computed here with numpy's FFT, for odd and even source sizes."""
    from oracle import pyoracle
    psf = W.gaussian_psf(7, 2.0)
    for (w, h) in [(31, 25), (30, 24)]:
        m = OracleModel(w, h)
        m.set_psf(psf)
        m.set_convolver("fft")
        m.add_profile("sersic", xcen=w / 2 + 0.3, ycen=h / 2 - 0.2, re=3, nser=1.5, convolve=True)
        got, _ = m.evaluate()
        # source image: the same model unconvolved on the padded grid
        dw, dh = m.drawing_dims()
        u = OracleModel(dw, dh)
        u.add_profile("sersic", xcen=w / 2 + 0.3 + (dw - w) / 2, ycen=h / 2 - 0.2 + (dh - h) / 2, re=3, nser=1.5)
        src, _ = u.evaluate()
        ext_w, ext_h = 2 * max(dw, 7), 2 * max(dh, 7)
        ext_src = np.zeros((ext_h, ext_w))
        ext_src[:dh, :dw] = src
        ext_krn = np.zeros((ext_h, ext_w))
        ky0, kx0 = (dh - 7) // 2, (dw - 7) // 2
        ext_krn[ky0:ky0 + 7, kx0:kx0 + 7] = psf / psf.sum()
        n = ext_w * ext_h
        conv = np.fft.irfft(np.fft.rfft(ext_src.ravel()) * np.fft.rfft(ext_krn.ravel()), n).reshape(ext_h, ext_w)
        ox = dw // 2 - (1 if (dw % 2 == 0 or 7 % 2 == 0) else 0)
        oy = dh // 2 - (1 if (dh % 2 == 0 or 7 % 2 == 0) else 0)
        full = conv[oy:oy + dh, ox:ox + dw]
        pad = 3
        expect = full[pad:pad + h, pad:pad + w]
        assert np.max(np.abs(got - expect)) <= 1e-12 * np.max(np.abs(expect))


@pytest.mark.parametrize("kind", ["chisq", "t", "pois"])
def test_other_likelihoods_restatement_matches_scipy(kind):
    """The oracle's chisq / t / pois likelihoods against scipy.stats' densities
    (the same closed forms R's dchisq and dt evaluate by saddle-point
    expansions)."""
    import scipy.stats as st
    from oracle.pyoracle import loglike_other
    r = np.random.Generator(np.random.PCG64(3))
    model = r.uniform(5, 50, size=(30, 40))
    sigma = r.uniform(0.5, 2, size=model.shape)
    image = model + r.standard_t(5, size=model.shape) * sigma * 1.3
    region = r.uniform(size=model.shape) < 0.9
    got = loglike_other(kind, image, sigma, model, region)
    x = ((image - model) / sigma)[region]
    if kind == "chisq":
        want = st.chi2.logpdf(np.sum(x * x), x.size)
    elif kind == "t":
        v = np.var(x, ddof=1)
        want = np.sum(st.t.logpdf(x, max(1.0, 2 * v / (v - 1))))
    else:
        im, md, sg = image[region], model[region], sigma[region]
        s = np.max(np.abs(im) / sg ** 2)
        if s < 0.1 or s > 10:
            im, md = im * s, md * s
        want = -np.sum(md - im * np.log(md))
    assert got == pytest.approx(want, rel=1e-12)
