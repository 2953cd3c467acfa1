"""Catalogue batches (pf_catalogue_*): galaxies of uneven image and PSF sizes,
1-3 profiles of any radial kind each, evaluated together.  Each galaxy's logL
and gradient must equal what the same galaxy gives alone through the model
API, and the gradient must match FP64 finite differences of the plain form."""
import numpy as np
import pytest

from profit_b200 import PF_FP32, Model
from profit_b200 import workloads as W
from profit_b200.catalogue import Catalogue, grad_names

pytestmark = pytest.mark.gpu


def _model(gal, precision=None):
    side = gal["side"]
    m = Model(side, side) if precision is None else Model(side, side, precision=precision)
    m.set_magzero(gal["magzero"])
    m.set_psf(gal["psf"])
    for kind, params in gal["profiles"]:
        m.add_profile(kind, convolve=True, **params)
    return m


def _refs(gal):
    return [(i, k) for i, (kind, _) in enumerate(gal["profiles"]) for k in grad_names(kind)]


def _catalogue_case(n=12, seed_tag=61):
    gals = W.catalogue(n, seed_tag=seed_tag, side_range=(24, 90))
    r = np.random.Generator(np.random.PCG64(5))
    for g in gals:
        img, _ = _model(g).evaluate()
        sigma = r.uniform(0.5, 2.0, size=img.shape)
        g["data"] = img + r.normal(size=img.shape) * sigma
        g["sigma"] = sigma
        # evaluate a little away from the truth so gradients carry signal
        g["profiles"] = [(k, {**p, "xcen": p["xcen"] + 0.3, "mag": p["mag"] + 0.05}) for k, p in g["profiles"]]
    return gals


def test_catalogue_matches_single_galaxies():
    gals = _catalogue_case()
    cat = Catalogue(magzero=gals[0]["magzero"])
    for g in gals:
        cat.add_galaxy(g["data"], g["sigma"], g["psf"], g["profiles"])
    ll, grads = cat.loglike_grad()
    # a second evaluation reuses the uploaded inputs; FP32 cells are added to
    # their pixels atomically in no fixed order, so runs agree to FP32 rounding
    # (these galaxies sit away from their truth, so large residuals amplify
    # FP32 rounding; 1e-5 is the FP32 form's accuracy bound)
    ll2, grads2 = cat.loglike_grad()
    np.testing.assert_allclose(ll2, ll, rtol=1e-5)
    for g, l, gr in zip(gals, ll, grads):
        m = _model(g, PF_FP32)
        m.set_data(g["data"], g["sigma"])
        l1, g1 = m.loglike_grad(_refs(g))
        assert l == pytest.approx(l1, rel=1e-5)
        np.testing.assert_allclose(gr, g1, rtol=1e-5, atol=1e-5 * np.max(np.abs(g1)))
        m64 = _model(g)
        m64.set_data(g["data"], g["sigma"])
        assert l == pytest.approx(m64.loglike(), rel=1e-5)


def test_catalogue_gradient_matches_fd64():
    gals = _catalogue_case(n=4, seed_tag=62)
    cat = Catalogue(magzero=gals[0]["magzero"])
    for g in gals:
        cat.add_galaxy(g["data"], g["sigma"], g["psf"], g["profiles"])
    _, grads = cat.loglike_grad()
    for g, gr in zip(gals, grads):
        m64 = _model(g)
        m64.set_data(g["data"], g["sigma"])
        refs = _refs(g)
        _, g6 = m64.loglike_grad_fd(refs, rel_step=1e-6)
        _, g5 = m64.loglike_grad_fd(refs, rel_step=1e-5)
        scale = np.linalg.norm(g6)
        err = np.minimum(np.abs(gr - g6), np.abs(gr - g5)) / scale
        spread = 2 * np.abs(g6 - g5) / scale  # FD unsteadiness (decision flips inside +-h)
        assert np.all(err <= np.maximum(1e-5, spread)), list(zip(refs, g6, g5, gr))


def test_catalogue_rejects_bad_input():
    from profit_b200._capi import InvalidParameter, UnknownParameter
    cat = Catalogue()
    psf = W.gaussian_psf(9, 2.0)
    with pytest.raises(InvalidParameter):
        cat.add_galaxy(np.zeros((10, 10)), np.zeros((10, 10)), psf, [])  # sigma must be positive
    with pytest.raises(UnknownParameter):
        cat.add_galaxy(np.zeros((10, 10)), np.ones((10, 10)), psf, [("sersic", {"fwhm": 2.0})])
    with pytest.raises(InvalidParameter):
        cat.add_galaxy(np.zeros((10, 10)), np.ones((10, 10)), psf, [("sky", {"bg": 1.0})])


def test_catalogue_replay_matches_first_call():
    """The second call replays the first call's recorded launch sequence (one
    graph for the prologue and every chunk); its results equal a fresh
    catalogue's first, eager call to FP32 rounding, and a third call gives
    the second's."""
    gals = _catalogue_case(n=10, seed_tag=64)
    out = []
    for _ in range(2):
        cat = Catalogue(magzero=gals[0]["magzero"])
        for g in gals:
            cat.add_galaxy(g["data"], g["sigma"], g["psf"], g["profiles"])
        out.append(cat)
    ll0, g0 = out[0].loglike_grad()          # eager (recorded afterwards)
    ll1, g1 = out[1].loglike_grad()          # eager, another catalogue
    ll2, g2 = out[1].loglike_grad()          # replayed
    ll3, g3 = out[1].loglike_grad()          # replayed again
    # (FP32 cells are added to their pixels atomically, in no fixed order)
    np.testing.assert_allclose(ll1, ll0, rtol=1e-6)
    np.testing.assert_allclose(ll2, ll1, rtol=1e-6)
    np.testing.assert_allclose(ll3, ll2, rtol=1e-6)
    for a, b, c in zip(g1, g2, g3):
        np.testing.assert_allclose(b, a, rtol=1e-5, atol=1e-6 * np.max(np.abs(a)))
        np.testing.assert_allclose(c, b, rtol=1e-5, atol=1e-6 * np.max(np.abs(b)))


def test_catalogue_set_values_matches_a_fresh_catalogue():
    """A sampler's step over a catalogue: new values for every profile
    (pf_catalogue_set_values) keep the images, batching and recorded launches,
    and give what a catalogue built with those values gives; bad values are
    refused without changing anything."""
    from profit_b200._capi import InvalidParameter
    gals = _catalogue_case(n=10, seed_tag=65)
    cat = Catalogue(magzero=gals[0]["magzero"])
    for g in gals:
        cat.add_galaxy(g["data"], g["sigma"], g["psf"], g["profiles"])
    cat.loglike_grad()
    cat.loglike_grad()  # recorded and replayed with the first values
    v0 = cat.values()
    r = np.random.Generator(np.random.PCG64(7))
    moved = []
    for g in gals:
        profs = []
        for kind, p in g["profiles"]:
            q = dict(p)
            q["xcen"] += r.uniform(-0.5, 0.5)
            q["mag"] += r.uniform(-0.1, 0.1)
            q["axrat"] = min(1.0, max(0.1, q["axrat"] * r.uniform(0.9, 1.1)))
            if kind in ("sersic", "coresersic"):
                q["nser"] *= r.uniform(0.9, 1.1)  # may cross nser = 1 (the centre cusp)
            profs.append((kind, q))
        moved.append(dict(g, profiles=profs))
    fresh = Catalogue(magzero=gals[0]["magzero"])
    for g in moved:
        fresh.add_galaxy(g["data"], g["sigma"], g["psf"], g["profiles"])
    v1 = fresh.values()
    assert v1.shape == v0.shape
    bad = v1.copy()
    bad[4] = 1.5  # axrat > 1
    with pytest.raises(InvalidParameter):
        cat.set_values(bad)
    np.testing.assert_array_equal(cat.values(), v0)
    cat.set_values(v1)
    np.testing.assert_array_equal(cat.values(), v1)
    ll_f, g_f = fresh.loglike_grad()
    for _ in range(2):  # the recorded call replayed with the new values
        ll, gr = cat.loglike_grad()
        # FP32 cells are added to their pixels atomically in no fixed order (and
        # the two catalogues run their chunks on different lanes); away from
        # the truth large residuals amplify that rounding: the FP32 bound
        np.testing.assert_allclose(ll, ll_f, rtol=1e-5)
        for a, b in zip(gr, g_f):
            np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-5 * np.max(np.abs(b)))


def _uneven_shapes_case():
    """Galaxies whose images and PSFs are not square, and PSFs of even side,
    beside square ones; two galaxies per shape so every batch holds several."""
    r = np.random.Generator(np.random.PCG64(11))
    shapes = [((40, 40), (15, 15)), ((64, 48), (16, 16)), ((33, 57), (21, 17)), ((90, 90), (31, 31)),
              ((120, 100), (45, 45))]
    gals = []
    for (w, h), (pw, ph) in shapes:
        for _ in range(2):
            yy, xx = np.mgrid[0:ph, 0:pw]
            psf = np.exp(-0.5 * (((xx - (pw - 1) / 2) / 1.6) ** 2 + ((yy - (ph - 1) / 2) / 1.9) ** 2))
            profs = W.catalogue_galaxy_profiles(r, min(w, h))
            profs = [(k, {**p, "xcen": p["xcen"] * w / min(w, h), "ycen": p["ycen"] * h / min(w, h)})
                     for k, p in profs]
            sigma = r.uniform(0.5, 2.0, size=(h, w))
            data = r.normal(size=(h, w)) * sigma
            gals.append(dict(w=w, h=h, psf=psf / psf.sum(), profiles=profs, data=data, sigma=sigma))
    return gals


def test_catalogue_fft_convolution_matches_brute_force():
    """The catalogue's FFT convolver (each galaxy's PSF spectrum, FP64
    transforms, the brute-force kernels' geometry) gives the brute-force
    logL and gradients to FP32 rounding, on square and non-square images and
    PSFs (even sides included); "auto" keeps one of the two per batch."""
    gals = _uneven_shapes_case()
    res = {}
    for mode in ("brute", "fft", "auto"):
        cat = Catalogue(magzero=30.0)
        cat.set_convolver(mode)
        for g in gals:
            cat.add_galaxy(g["data"], g["sigma"], g["psf"], g["profiles"])
        res[mode] = cat.loglike_grad()
        res[mode + "_replayed"] = cat.loglike_grad()  # the recorded call
        fft, n = cat.convolvers()
        assert n == 5
        assert fft == {"brute": 0, "fft": 5}.get(mode, fft)
    ll_b, g_b = res["brute"]
    for key in ("fft", "fft_replayed", "auto", "auto_replayed", "brute_replayed"):
        ll, gr = res[key]
        np.testing.assert_allclose(ll, ll_b, rtol=1e-5, err_msg=key)
        for a, b in zip(gr, g_b):
            np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-5 * np.max(np.abs(b)), err_msg=key)


def test_catalogue_fft_convolution_matches_single_galaxies():
    """Through FFTs, each galaxy's logL and gradient equal what it gives
    alone through the model API (brute-force convolution) and the FP64 form."""
    gals = _catalogue_case(n=8, seed_tag=66)
    cat = Catalogue(magzero=gals[0]["magzero"])
    cat.set_convolver("fft")
    for g in gals:
        cat.add_galaxy(g["data"], g["sigma"], g["psf"], g["profiles"])
    ll, grads = cat.loglike_grad()
    assert cat.convolvers()[0] == cat.convolvers()[1]
    for g, l, gr in zip(gals, ll, grads):
        m = _model(g, PF_FP32)
        m.set_data(g["data"], g["sigma"])
        l1, g1 = m.loglike_grad(_refs(g))
        assert l == pytest.approx(l1, rel=1e-5)
        np.testing.assert_allclose(gr, g1, rtol=1e-5, atol=1e-5 * np.max(np.abs(g1)))
        m64 = _model(g)
        m64.set_data(g["data"], g["sigma"])
        assert l == pytest.approx(m64.loglike(), rel=1e-5)


def test_catalogue_convolver_names():
    from profit_b200._capi import InvalidParameter
    cat = Catalogue()
    for name in ("auto", "brute", "fft"):
        cat.set_convolver(name)
    with pytest.raises(InvalidParameter):
        cat.set_convolver("brute-old")
