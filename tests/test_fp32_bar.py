"""The FP32 + adjoint form against the gradient oracle on the configurations
the benchmark times (needs a B200 and the compiled reference).

The bar: logL within 1e-5 relative of the FP64 oracle, and the gradient
within 1e-5 relative.  The gradient oracle is FP64 central differences of
the compiled reference (tests/fdref.py), at relative steps 1e-8 ... 1e-6
(C4: 1e-7, 1e-6), each component compared with the step that agrees best
among those at which no subsampling decision, resolution or rscale_max
changes between theta - h and theta + h (restatement decision log and the
reference's PROFIT_DEBUG counters).

Gradient errors are stated three ways (fdref.gradient_errors): per component
relative to its own size ("own"), the vector's relative error ("norm"), and
per component relative to the gradient's norm ("of_norm").  On the single
models (C1-C3) every component meets 1e-5 on its own size.  Where a component
is a small difference of large terms (a catalogue galaxy of a few pixels at
S/N in the thousands, where d logL / d rt or d logL / d ang is 1e-3 of the
gradient's norm), FP32 tangents and FD's own roundoff cannot resolve it to
1e-5 of itself; there the bar is the vector's relative error and each
component's error relative to the norm.
"""
import os

import numpy as np
import pytest

from fdref import gradient_errors, ref_fd_gradient, _decision_log, _same_log, _with
from oracle.pyoracle import OracleModel
from profit_b200 import PF_FP32, PF_FP64, Model
from profit_b200 import workloads as W

pytestmark = pytest.mark.gpu

BAR = 1e-5


def _data(wl):
    m64 = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m64.evaluate()
    return W.make_data(wl, truth)


def _check(tag, ll_ad, g_ad, fd, own=True):
    ll_rel = abs(ll_ad - fd["loglike"]) / abs(fd["loglike"])
    e = gradient_errors(g_ad, fd)
    assert ll_rel <= BAR, (tag, ll_rel)
    assert e["usable"].sum() >= len(g_ad) - 2, (tag, "too many components with a decision flip at every step")
    assert e["norm"] <= BAR, (tag, e["norm"])
    assert np.all(e["of_norm"] <= BAR), (tag, e["of_norm"].max())
    if own:
        assert np.all(e["own"] <= BAR), (tag, list(zip(g_ad, e["ref"], e["own"])))


@pytest.mark.parametrize("seed", [5, 6])
def test_c1_single_sersic(seed):
    """C1: one Sersic on 100x100 with a 25x25 Gaussian PSF, 8 parameters
    (magzero 25 so the source stands above the unit noise: at magzero 0 the
    configuration's mag 15 is a total flux of 1e-6 and the gradient is below
    FD's roundoff)."""
    wl = W.single_sersic()
    wl["magzero"] = 25.0
    image, sigma = _data(wl)
    w2 = W.perturbed(wl, seed=seed, scale=0.02)
    m = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), w2)
    m.set_data(image, sigma)
    ll, g = m.loglike_grad(w2["grad"])
    fd = ref_fd_gradient(wl, w2["profiles"], image, sigma, w2["grad"], (1e-8, 1e-7, 1e-6))
    _check(f"C1 seed {seed}", ll, g, fd)


@pytest.mark.parametrize("seed", [5, 6])
def test_c2_bulge_disk_point_source(seed):
    """C2 (the headline): 400x400 bulge + disk + point source, 51x51 Moffat
    PSF, brute force, all 17 parameters, one call as the benchmark makes it
    and a graph replay."""
    wl = W.bulge_disk_ps()
    image, sigma = _data(wl)
    w2 = W.perturbed(wl, seed=seed, scale=0.02)
    m = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    m.set_data(image, sigma)
    vals = [w2["profiles"][i][1][k] for (i, k) in w2["grad"]]
    m.set_parameters(w2["grad"], vals)
    m.loglike_grad(w2["grad"])
    ll, g = m.loglike_grad(w2["grad"])  # replayed from the captured graph
    fd = ref_fd_gradient(wl, w2["profiles"], image, sigma, w2["grad"], (1e-8, 1e-7, 1e-6))
    _check(f"C2 seed {seed}", ll, g, fd)


def test_c3_sampler_batch_rows():
    """C3: the sampler batch's model (one Sersic, 200x200, 31x31 Gaussian
    PSF, proposals init + N(0, 0.05 |init|)), 8 proposals in one
    pf_model_loglike_grad_batch call, each row against the oracle
    (magzero 25 as in C1)."""
    wl, vals = W.sampler_batch(8)
    wl["magzero"] = 25.0
    image, sigma = _data(wl)
    mb = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    mb.set_data(image, sigma)
    ll_b, g_b = mb.loglike_grad_batch(wl["grad"], vals)
    for b in range(len(vals)):
        profs = [(n, dict(p)) for n, p in wl["profiles"]]
        for (pi, k), v in zip(wl["grad"], vals[b]):
            profs[pi][1][k] = float(v)
        fd = ref_fd_gradient(wl, profs, image, sigma, wl["grad"], (1e-8, 1e-7, 1e-6))
        _check(f"C3 row {b}", ll_b[b], g_b[b], fd)


def _catalogue_galaxies():
    """16 galaxies of the uneven catalogue with sides 32-512 and PSFs 15-65,
    the first forced to a 512x512 image with a 65x65 PSF; data at the truth,
    the model a little away from it."""
    gals = W.catalogue(16, seed_tag=63, side_range=(32, 512))
    gals[0]["side"] = 512
    gals[0]["psf"] = W.moffat_psf(65, 3.0, 2.5)
    gals[0]["profiles"] = W.catalogue_galaxy_profiles(np.random.Generator(np.random.PCG64(3)), 512)
    r = np.random.Generator(np.random.PCG64(5))
    for g in gals:
        m = Model(g["side"], g["side"])
        m.set_magzero(g["magzero"])
        m.set_psf(g["psf"])
        for kind, p in g["profiles"]:
            m.add_profile(kind, convolve=True, **p)
        img, _ = m.evaluate()
        sg = r.uniform(0.5, 2.0, size=img.shape)
        g["data"] = img + r.normal(size=img.shape) * sg
        g["sigma"] = sg
        g["profiles"] = [(k, {**p, "xcen": p["xcen"] + 0.3, "mag": p["mag"] + 0.05}) for k, p in g["profiles"]]
    return gals


def test_c4_uneven_catalogue():
    """C4: 16 galaxies (sides 32-512, PSFs 15-65, 1-3 components of the six
    radial kinds) in one pf_catalogue_loglike_grad call, every galaxy against
    the oracle.  Components are compared with the norm of their galaxy's
    gradient (module docstring)."""
    from profit_b200.catalogue import Catalogue, grad_names
    gals = _catalogue_galaxies()
    sides = [g["side"] for g in gals]
    psfs = [g["psf"].shape[0] for g in gals]
    assert max(sides) == 512 and min(sides) < 48 and max(psfs) == 65 and min(psfs) <= 21
    cat = Catalogue(magzero=gals[0]["magzero"])
    for g in gals:
        cat.add_galaxy(g["data"], g["sigma"], g["psf"], g["profiles"])
    ll, grads = cat.loglike_grad()
    for gi, (g, gr) in enumerate(zip(gals, grads)):
        wlg = dict(width=g["side"], height=g["side"], magzero=g["magzero"], psf=g["psf"])
        profs = [(k, {**p, "convolve": True}) for k, p in g["profiles"]]
        refs = [(i, k) for i, (kind, _) in enumerate(g["profiles"]) for k in grad_names(kind)]
        fd = ref_fd_gradient(wlg, profs, g["data"], g["sigma"], refs, (1e-7, 1e-6))
        _check(f"C4 galaxy {gi}", ll[gi], gr, fd, own=False)


def test_c5_large_field():
    """C5 at 1000x1000 with 50 Sersic components and the 101x101 Moffat PSF
    (FFT convolver): the plain FP64 image against the oracle's restatement to
    1e-12, and the FP32 recomputing adjoint of four components (32
    parameters) against FP64 central differences.  At this size the FD
    values come from the plain FP64 form (equal to the restatement's image to
    1e-12, asserted first), with the flip check of the restatement's
    decision log for the varied profile."""
    from profit_b200._capi import PF_ADJOINT_RECOMPUTE
    wl = W.large_field(n_profiles=50, width=1000, height=1000, psf_size=101)
    ora = W.configure(OracleModel(wl["width"], wl["height"], threads=os.cpu_count() or 1), wl)
    expect, _ = ora.evaluate()
    m = W.configure(Model(wl["width"], wl["height"]), wl)
    got, _ = m.evaluate()
    assert float(np.max(np.abs(got - expect)) / np.max(np.abs(expect))) <= 1e-12
    image, sigma = W.make_data(wl, expect)
    w2 = W.perturbed(wl, seed=9, scale=0.01)
    refs = [(i, k) for (i, k) in w2["grad"] if i in (0, 7, 21, 40)]
    mp = W.configure(Model(wl["width"], wl["height"]), w2)
    mp.set_data(image, sigma)
    ll64 = mp.loglike()
    grads, flips = {}, {}
    base = {pi: _decision_log(wl, w2["profiles"], pi) for pi in (0, 7, 21, 40)}
    for s in (1e-8, 1e-7, 1e-6):
        _, grads[s] = mp.loglike_grad_fd(refs, rel_step=s)
        fl = np.zeros(len(refs), bool)
        for j, (pi, k) in enumerate(refs):
            v = w2["profiles"][pi][1][k]
            h = s * max(abs(v), 1.0)
            fl[j] = not (_same_log(_decision_log(wl, _with(w2["profiles"], {pi: {k: v + h}}), pi), base[pi]) and
                         _same_log(_decision_log(wl, _with(w2["profiles"], {pi: {k: v - h}}), pi), base[pi]))
        flips[s] = fl
    mp.set_precision(PF_FP32)
    mp.set_adjoint_mode(PF_ADJOINT_RECOMPUTE)
    ll, g = mp.loglike_grad(refs)
    fd = {"loglike": ll64, "grad": grads, "flipped": flips}
    # the cusp of profile 21 (n = 5.2) flips decisions at every step in x and y
    e = gradient_errors(g, fd)
    assert abs(ll - ll64) / abs(ll64) <= BAR
    assert e["usable"].sum() >= len(refs) - 4
    assert e["norm"] <= BAR and np.all(e["of_norm"] <= BAR), (e["norm"], e["of_norm"].max())
