"""Parity of the sm_100a library against the oracle (needs a B200).

Plain FP64 form: images within 1e-12 (relative to the image maximum) of the
compiled reference, the same subsampling decision for every pixel as the
restatement, the same per-level counts as libprofit's PROFIT_DEBUG counters,
and the same "norm" log-likelihood to 1e-12 relative.

FP32 form: images within 1e-5 of the FP64 form; the adjoint gradient within
the tolerances stated in each test of FP64 central finite differences.
"""
import numpy as np
import pytest

from oracle.pyoracle import OracleModel, RefModel, loglike_norm
from profit_b200 import PF_FP32, PF_FP64, InvalidParameter, Model, UnknownParameter
from profit_b200 import workloads as W

from test_oracle import PROFILE_CASES

pytestmark = pytest.mark.gpu

IMG_TOL = 1e-12


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("case", range(len(PROFILE_CASES)))
def test_render_fp64_matches_reference(case):
    name, params = PROFILE_CASES[case]
    ref = RefModel(100, 100)
    ref.add_profile(name, **params)
    expect, _ = ref.evaluate()
    m = Model(100, 100)
    m.set_debug(True)
    m.add_profile(name, **params)
    got, off = m.evaluate()
    assert off == (0, 0)
    assert _rel(got, expect) <= IMG_TOL
    # decisions: pixel by pixel against the restatement, per level against PROFIT_DEBUG
    ora = OracleModel(100, 100)
    ora.add_profile(name, **params)
    ora.evaluate()
    assert np.array_equal(m.decisions(0), ora.decisions(0))
    assert m.level_counts(0) == ora.level_counts(0)
    assert m.evaluation_counts(0)[0] == ora.evaluations(0)
    dbg = RefModel(100, 100, debug=True)
    dbg.set_omp_threads(1)
    dbg.add_profile(name, **params)
    dbg.evaluate()
    assert m.level_counts(0) == dbg.integrations(0)


@pytest.mark.parametrize("wl", [W.single_sersic(), W.single_sersic(seed_tag=11), W.bulge_disk_ps()],
                         ids=["single_sersic", "single_sersic_b", "bulge_disk_ps"])
def test_workload_fp64_image_and_loglike(wl):
    ref = W.configure(RefModel(wl["width"], wl["height"]), wl)
    ref.set_omp_threads(8)
    ref.set_convolver("brute", 8)
    expect, _ = ref.evaluate()
    m = W.configure(Model(wl["width"], wl["height"]), wl)
    got, _ = m.evaluate()
    assert got.shape == expect.shape
    assert _rel(got, expect) <= IMG_TOL
    image, sigma = W.make_data(wl, expect)
    m.set_data(image, sigma)
    ll = m.loglike()
    assert ll == pytest.approx(loglike_norm(image, sigma, expect), rel=IMG_TOL)


def test_sky_and_psf_point_source_fp64():
    psf = W.moffat_psf(15, 3.0, 2.5)
    out = []
    for M in (RefModel, Model):
        m = M(60, 50)
        m.set_psf(psf)
        m.add_profile("sersic", xcen=30, ycen=25, re=4, nser=2, convolve=True)
        m.add_profile("sky", bg=0.25)
        m.add_profile("psf", xcen=12.3, ycen=40.6, mag=14)
        m.add_profile("psf", xcen=-3.0, ycen=55.0, mag=13)  # partly outside the image
        out.append(m.evaluate()[0])
    assert _rel(out[1], out[0]) <= IMG_TOL


def test_null_convolver_and_rough():
    wl = W.single_sersic(seed_tag=3)
    out = []
    for M in (RefModel, Model):
        m = W.configure(M(wl["width"], wl["height"]), wl)
        m.set_convolver("null")
        m.add_profile("sersic", xcen=20.5, ycen=70.2, re=3, nser=1.5, rough=True)
        out.append(m.evaluate()[0])
    assert _rel(out[1], out[0]) <= IMG_TOL


def test_finesampling_downsampled():
    wl = W.single_sersic(seed_tag=4, width=60, height=50, psf_size=11)
    out = []
    for M in (RefModel, Model):
        m = W.configure(M(wl["width"], wl["height"]), wl)
        m.set_finesampling(3)
        m.set_return_finesampled(False)
        out.append(m.evaluate()[0])
    assert out[1].shape == out[0].shape == (50, 60)
    assert _rel(out[1], out[0]) <= IMG_TOL


@pytest.mark.parametrize("w,h,psf_size", [(31, 25, 7), (30, 24, 7), (64, 51, 10), (120, 100, 25)])
def test_fft_convolver_fp64_matches_restated_geometry(w, h, psf_size):
    """FFTConvolver (convolve.cpp:233-312) on the GPU against the oracle's
    restatement of the same linear convolution and crop offset, including
    even image and even PSF sizes, to 1e-12 of the image maximum."""
    psf = W.gaussian_psf(psf_size, 2.0) if psf_size % 2 else W.moffat_psf(psf_size, 2.5, 2.0)
    out = []
    for M in (OracleModel, Model):
        m = M(w, h)
        m.set_psf(psf)
        m.set_convolver("fft")
        m.add_profile("sersic", xcen=w / 2 + 0.3, ycen=h / 2 - 0.2, re=3, nser=1.5, convolve=True)
        m.add_profile("moffat", xcen=w / 3, ycen=h / 3, fwhm=2.0, con=3.0)  # not convolved
        out.append(m.evaluate()[0])
    assert _rel(out[1], out[0]) <= IMG_TOL


def test_fft_adjoint_gradient_matches_fd64():
    wl = W.bulge_disk_ps(width=160, height=150, psf_size=25)
    wl["convolver"] = "fft"
    m, w2 = _gradient_case(wl, 0.02)
    _, g_fd = m.loglike_grad_fd(w2["grad"], rel_step=1e-7)
    m.set_precision(PF_FP32)
    _, g_ad = m.loglike_grad(w2["grad"])
    err = np.max(np.abs(g_ad - g_fd)) / np.max(np.abs(g_fd))
    assert err <= 1e-5, list(zip(w2["grad"], g_fd, g_ad))


def test_recompute_adjoint_matches_stored_tangents():
    """The two adjoint forms (stored tangent planes / recomputed tangents with
    recorded decisions) give the same gradient."""
    from profit_b200._capi import PF_ADJOINT_RECOMPUTE, PF_ADJOINT_STORE
    wl = W.bulge_disk_ps(width=200, height=180, psf_size=25)
    m, w2 = _gradient_case(wl, 0.02)
    m.set_precision(PF_FP32)
    m.set_adjoint_mode(PF_ADJOINT_STORE)
    ll_s, g_s = m.loglike_grad(w2["grad"])
    m.set_adjoint_mode(PF_ADJOINT_RECOMPUTE)
    ll_r, g_r = m.loglike_grad(w2["grad"])
    # two runs of the FP32 render add sub-pixel cells in different orders
    assert ll_r == pytest.approx(ll_s, rel=1e-6)
    np.testing.assert_allclose(g_r, g_s, rtol=1e-5, atol=1e-6 * np.max(np.abs(g_s)))


def test_recompute_adjoint_tile_lists_match_stored_tangents():
    """Models with many profiles take per-tile profile lists in the
    recomputing adjoint (12 Sersics here): every component's gradient equals
    the stored-plane form's."""
    from profit_b200._capi import PF_ADJOINT_RECOMPUTE, PF_ADJOINT_STORE
    wl = W.large_field(n_profiles=12, width=240, height=200, psf_size=31)
    m = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m.evaluate()
    image, sigma = W.make_data(wl, truth)
    w2 = W.perturbed(wl, seed=11, scale=0.01)
    mp = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), w2)
    mp.set_data(image, sigma)
    refs = w2["grad"]
    mp.set_adjoint_mode(PF_ADJOINT_STORE)
    ll_s, g_s = mp.loglike_grad(refs)
    mp.set_adjoint_mode(PF_ADJOINT_RECOMPUTE)
    ll_r, g_r = mp.loglike_grad(refs)
    assert ll_r == pytest.approx(ll_s, rel=1e-6)
    np.testing.assert_allclose(g_r, g_s, rtol=1e-5, atol=1e-6 * np.max(np.abs(g_s)))


def test_large_field_fft_fp64_and_recompute_gradient():
    """A field of 12 Sersics (shape of the 2000x2000 / 200-component case at
    reduced size) with the FFT convolver: FP64 image against the restatement,
    recompute-adjoint gradient of two components against FP64 FD."""
    wl = W.large_field(n_profiles=12, width=240, height=200, psf_size=31)
    ora = W.configure(OracleModel(wl["width"], wl["height"]), wl)
    expect, _ = ora.evaluate()
    m = W.configure(Model(wl["width"], wl["height"]), wl)
    got, _ = m.evaluate()
    assert _rel(got, expect) <= IMG_TOL
    image, sigma = W.make_data(wl, expect)
    w2 = W.perturbed(wl, seed=9, scale=0.01)
    refs = [(i, k) for (i, k) in w2["grad"] if i in (0, 5)]
    mp = W.configure(Model(wl["width"], wl["height"]), w2)
    mp.set_data(image, sigma)
    # A subsampling decision that flips inside +-h puts a jump into a finite
    # difference; two step sizes guard against it (the adjoint differentiates
    # the quadrature with decisions held fixed).
    _, g_fd7 = mp.loglike_grad_fd(refs, rel_step=1e-7)
    _, g_fd6 = mp.loglike_grad_fd(refs, rel_step=1e-6)
    from profit_b200._capi import PF_ADJOINT_RECOMPUTE
    mp.set_precision(PF_FP32)
    mp.set_adjoint_mode(PF_ADJOINT_RECOMPUTE)
    _, g_ad = mp.loglike_grad(refs)
    scale = np.max(np.abs(g_fd7))
    err = np.minimum(np.abs(g_ad - g_fd7), np.abs(g_ad - g_fd6)) / scale
    assert np.all(err <= 1e-5), list(zip(refs, g_fd7, g_fd6, g_ad))


def test_errors_match_libprofit():
    m = Model(10, 10)
    with pytest.raises(InvalidParameter):
        m.add_profile("nonexistent")
    p = m.add_profile("sersic")
    with pytest.raises(UnknownParameter):
        p.parameter("fwhm", 3.0)
    p.parameter("axrat", 1.5)
    with pytest.raises(InvalidParameter, match="axrat > 1"):
        m.evaluate()
    p.parameter("axrat = 0.5")
    p.parameter("convolve", True)
    with pytest.raises(InvalidParameter, match="No psf provided"):
        m.evaluate()


@pytest.mark.parametrize("wl", [W.single_sersic(), W.bulge_disk_ps()], ids=["single_sersic", "bulge_disk_ps"])
def test_fp32_image_close_to_fp64(wl):
    m64 = W.configure(Model(wl["width"], wl["height"]), wl)
    a, _ = m64.evaluate()
    m32 = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    b, _ = m32.evaluate()
    assert _rel(b, a) <= 1e-5


# Number of FP32 convolution kernels the autotuner chooses from (render32.cu).
N_FP32_CONV_CANDIDATES = 33
# candidates 20-29 are compiled for one kernel height (51 or 31): they are
# tested with a PSF of that size
FIXED_HEIGHT_CANDIDATES = {20: 51, 21: 51, 22: 51, 23: 51, 24: 31, 25: 31, 26: 51, 27: 51, 28: 51, 29: 51}
# candidates from this index on run on the tensor cores (3xTF32 split
# products): their FP32-level sums differ from the FMA kernels' by a few
# 1e-7 of logL, so logL is compared at 1e-6 there
FIRST_TC_CONV_CANDIDATE = 30


@pytest.mark.parametrize("cand", range(N_FP32_CONV_CANDIDATES))
def test_every_fp32_convolution_candidate(cand, monkeypatch):
    """Each tile shape, column split and packed/unpacked FMA kernel gives the
    FP64 image to FP32 accuracy, and the same adjoint gradient, on odd sizes
    (partial tiles, kernel rows not a multiple of the unroll) and in a batch."""
    psf_size = FIXED_HEIGHT_CANDIDATES.get(cand, 21)
    wl = W.single_sersic(seed_tag=11, width=157, height=93, psf_size=psf_size)
    wl["magzero"] = 25.0
    m64 = W.configure(Model(wl["width"], wl["height"]), wl)
    ref, _ = m64.evaluate()
    image, sigma = W.make_data(wl, ref)
    refs = wl["grad"]
    props = [W.perturbed(wl, seed=300 + s, scale=0.03) for s in range(3)]
    vals = np.array([[p["profiles"][i][1][k] for (i, k) in refs] for p in props])

    base = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), props[0])
    base.set_data(image, sigma)
    ll0, g0 = base.loglike_grad(refs)

    monkeypatch.setenv("PF_CONV_FORCE", str(cand))
    m32 = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    img, _ = m32.evaluate()
    assert _rel(img, ref) <= 1e-6
    one = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), props[0])
    one.set_data(image, sigma)
    ll_rel = 1e-6 if cand >= FIRST_TC_CONV_CANDIDATE else 1e-7
    for _ in range(2):  # eager, then graph replay
        ll, g = one.loglike_grad(refs)
        assert ll == pytest.approx(ll0, rel=ll_rel)
        np.testing.assert_allclose(g, g0, rtol=1e-5, atol=1e-6 * np.max(np.abs(g0)))
    mb = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    mb.set_data(image, sigma)
    ll_b, g_b = mb.loglike_grad_batch(refs, vals)
    assert ll_b[0] == pytest.approx(ll0, rel=ll_rel)
    np.testing.assert_allclose(g_b[0], g0, rtol=1e-5, atol=1e-6 * np.max(np.abs(g0)))
    for s in (1, 2):
        p = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), props[s])
        p.set_data(image, sigma)
        ll, g = p.loglike_grad(refs)
        assert ll_b[s] == pytest.approx(ll, rel=1e-7)
        np.testing.assert_allclose(g_b[s], g, rtol=1e-5, atol=1e-6 * np.max(np.abs(g)))


def test_fp32_loglike_close_to_fp64():
    wl = W.bulge_disk_ps()
    m64 = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m64.evaluate()
    image, sigma = W.make_data(wl, truth)
    m64.set_data(image, sigma)
    ll64 = m64.loglike()
    m32 = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    m32.set_data(image, sigma)
    ll32 = m32.loglike()
    assert ll32 == pytest.approx(ll64, rel=1e-5)


def _gradient_case(wl, offset_scale):
    """Data drawn at the truth, model evaluated at a displaced point so the
    gradient is dominated by signal, not by noise."""
    m64 = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m64.evaluate()
    image, sigma = W.make_data(wl, truth)
    w2 = W.perturbed(wl, seed=5, scale=offset_scale)
    m = W.configure(Model(wl["width"], wl["height"]), w2)
    m.set_data(image, sigma)
    return m, w2


def test_graph_replay_matches_fresh_evaluation():
    """After the first call the FP32 pipeline is replayed from a CUDA graph;
    every proposal must give what a fresh model (first, eager call) gives."""
    wl = W.bulge_disk_ps(width=200, height=180, psf_size=25)
    m64 = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m64.evaluate()
    image, sigma = W.make_data(wl, truth)
    m = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    m.set_data(image, sigma)
    refs = wl["grad"]
    for s in range(4):
        w2 = W.perturbed(wl, seed=100 + s, scale=0.02)
        vals = [w2["profiles"][i][1][k] for (i, k) in refs]
        m.set_parameters(refs, vals)
        ll, g = m.loglike_grad(refs)
        fresh = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), w2)
        fresh.set_data(image, sigma)
        ll_f, g_f = fresh.loglike_grad(refs)
        # FP32 atomics accumulate sub-pixel sums in any order; at this
        # brightness that moves logL by ~1e-8 relative between runs
        assert ll == pytest.approx(ll_f, rel=1e-7)
        np.testing.assert_allclose(g, g_f, rtol=1e-5, atol=1e-6 * np.max(np.abs(g_f)))
        t = m.last_timings()
        assert t[0] > 0 and t[0] < 1e3


def test_batch_matches_single_proposals():
    """A batch of proposals gives, row by row, what one-proposal calls give;
    an invalid proposal (axrat > 1) yields -inf without failing the call."""
    wl = W.single_sersic(width=120, height=110, psf_size=15)
    wl["magzero"] = 25.0
    m = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m.evaluate()
    image, sigma = W.make_data(wl, truth)
    refs = wl["grad"]
    props = [W.perturbed(wl, seed=200 + s, scale=0.05) for s in range(7)]
    vals = np.array([[p["profiles"][i][1][k] for (i, k) in refs] for p in props])
    vals[3, refs.index((0, "axrat"))] = 1.5
    mb = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    mb.set_data(image, sigma)
    ll_b, g_b = mb.loglike_grad_batch(refs, vals)
    assert np.isneginf(ll_b[3]) and np.all(g_b[3] == 0)
    for s in range(7):
        if s == 3:
            continue
        one = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), props[s])
        one.set_data(image, sigma)
        ll, g = one.loglike_grad(refs)
        assert ll_b[s] == pytest.approx(ll, rel=1e-7)
        np.testing.assert_allclose(g_b[s], g, rtol=1e-5, atol=1e-6 * np.max(np.abs(g)))


def test_large_batch_matches_single_proposals():
    """Batches above 1024 (proposal, parameter) pairs assemble the gradient in
    their own launch, small ones inside the tangent reduction; both give what
    one-proposal calls give."""
    wl = W.single_sersic(width=96, height=90, psf_size=15)
    wl["magzero"] = 25.0
    m = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m.evaluate()
    image, sigma = W.make_data(wl, truth)
    refs = wl["grad"]
    n = 1024 // len(refs) + 20
    props = [W.perturbed(wl, seed=300 + s, scale=0.05) for s in range(n)]
    vals = np.array([[p["profiles"][i][1][k] for (i, k) in refs] for p in props])
    mb = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    mb.set_data(image, sigma)
    ll_b, g_b = mb.loglike_grad_batch(refs, vals)
    assert np.all(np.isfinite(ll_b))
    for s in (0, n // 2, n - 1):
        one = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), props[s])
        one.set_data(image, sigma)
        ll, g = one.loglike_grad(refs)
        assert ll_b[s] == pytest.approx(ll, rel=1e-7)
        np.testing.assert_allclose(g_b[s], g, rtol=1e-5, atol=1e-6 * np.max(np.abs(g)))


def test_adjoint_gradient_matches_fd64():
    """The headline model against FD of the plain FP64 form (the compiled
    reference's FD with decision checks is in test_fp32_bar.py): logL to
    1e-5, every component to 1e-5 of its own size, the closer of two steps."""
    wl = W.bulge_disk_ps()
    m, w2 = _gradient_case(wl, 0.02)
    ll_fd, g7 = m.loglike_grad_fd(w2["grad"], rel_step=1e-7)
    _, g8 = m.loglike_grad_fd(w2["grad"], rel_step=1e-8)
    m.set_precision(PF_FP32)
    ll_ad, g_ad = m.loglike_grad(w2["grad"])
    assert ll_ad == pytest.approx(ll_fd, rel=1e-5)
    err = np.minimum(np.abs(g_ad - g7), np.abs(g_ad - g8)) / np.abs(g7)
    assert np.all(err <= 1e-5), list(zip(w2["grad"], g7, g8, g_ad))


# One boxy profile of each kind without a closed-form luminosity derivative,
# all of its parameters in the gradient.
SHAPE_GRADIENT_CASES = {
    "ferrer": dict(rout=14.0, a=1.5, b=0.5),
    "coresersic": dict(re=9.0, rb=2.5, nser=2.5, a=3.0, b=0.6),
    "king": dict(rc=3.0, rt=18.0, a=2.0),
    "brokenexp": dict(h1=6.0, h2=3.0, rb=9.0, a=1.0),
}


@pytest.mark.parametrize("kind", sorted(SHAPE_GRADIENT_CASES))
def test_shape_gradients_of_every_profile_kind(kind):
    """FP32 adjoint gradient of every parameter of a Ferrer, core-Sersic, King
    or broken-exponential profile (box included) against FP64 central
    differences of the plain form; two FD steps guard against subsampling
    decisions that flip inside +-h."""
    shape = SHAPE_GRADIENT_CASES[kind]
    truth = dict(xcen=40.3, ycen=34.8, mag=17.0, ang=32.0, axrat=0.7, box=0.15, convolve=True, **shape)
    wl = dict(name=kind, width=80, height=70, magzero=25.0, psf=W.gaussian_psf(15, 2.5), convolver="brute",
              profiles=[(kind, truth)], sigma_range=(1.0, 1.0), seed_tag=41,
              grad=[(0, k) for k in ["xcen", "ycen", "mag", "ang", "axrat", "box"] + list(shape)])
    m64 = W.configure(Model(wl["width"], wl["height"]), wl)
    img, _ = m64.evaluate()
    image, sigma = W.make_data(wl, img)
    w2 = W.perturbed(wl, seed=9, scale=0.02)
    m = W.configure(Model(wl["width"], wl["height"]), w2)
    m.set_data(image, sigma)
    refs = w2["grad"]
    _, g6 = m.loglike_grad_fd(refs, rel_step=1e-6)
    _, g5 = m.loglike_grad_fd(refs, rel_step=1e-5)
    m.set_precision(PF_FP32)
    _, g = m.loglike_grad(refs)
    scale = np.max(np.abs(g6))
    err = np.minimum(np.abs(g - g6), np.abs(g - g5)) / scale
    # Where the reference itself is unsteady (the core-Sersic r^-b cusp flips
    # sub-cell decisions between +-h, so the two FD steps disagree), the
    # adjoint must lie within that spread; everywhere else within 1e-5.
    spread = 2 * np.abs(g6 - g5) / scale
    assert np.all(err <= np.maximum(1e-5, spread)), list(zip(refs, g6, g5, g))
    assert np.sum(spread > 1e-5) <= 2


@pytest.mark.parametrize("kind", ["chisq", "t", "pois"])
def test_other_likelihoods_and_their_gradients(kind):
    """profitLikeModel's chisq, t (dof from the residual variance) and pois
    likelihoods: the FP64 value against the oracle's restatement, the FP32
    value against FP64, and the FP32 adjoint gradient (through the t dof as
    well) against FP64 central differences."""
    from oracle.pyoracle import loglike_other
    wl = W.single_sersic(seed_tag=13, width=90, height=80, psf_size=15)
    wl["magzero"] = 25.0
    wl["profiles"] = wl["profiles"] + [("sky", dict(bg=5.0))]
    m64 = W.configure(Model(wl["width"], wl["height"]), wl)
    truth, _ = m64.evaluate()
    image, sigma = W.make_data(wl, truth)
    region = (np.random.Generator(np.random.PCG64(8)).uniform(size=image.shape) < 0.9).astype(np.uint8)
    w2 = W.perturbed(wl, seed=9, scale=0.02)
    m = W.configure(Model(wl["width"], wl["height"]), w2)
    m.set_data(image, sigma, region)
    m.set_likelihood(kind)
    ll64 = m.loglike()
    model_img, _ = m.evaluate()
    assert ll64 == pytest.approx(loglike_other(kind, image, sigma, model_img, region), rel=1e-11)
    refs = w2["grad"]
    _, g6 = m.loglike_grad_fd(refs, rel_step=1e-6)
    _, g5 = m.loglike_grad_fd(refs, rel_step=1e-5)
    m.set_precision(PF_FP32)
    ll32, g = m.loglike_grad(refs)
    assert ll32 == pytest.approx(ll64, rel=1e-5, abs=1e-6 * abs(ll64) + 1e-6)
    scale = np.max(np.abs(g6))
    err = np.minimum(np.abs(g - g6), np.abs(g - g5)) / scale
    spread = 2 * np.abs(g6 - g5) / scale
    assert np.all(err <= np.maximum(1e-5, spread)), list(zip(refs, g6, g5, g))
    if kind == "t":
        vals = np.array([[p["profiles"][i][1][k] for (i, k) in refs] for p in
                         [W.perturbed(wl, seed=30 + s, scale=0.02) for s in range(3)]])
        ll_b, g_b = m.loglike_grad_batch(refs, vals)
        for s in range(3):
            m.set_parameters(refs, vals[s])
            l1, g1 = m.loglike_grad(refs)
            assert ll_b[s] == pytest.approx(l1, rel=1e-7)
            np.testing.assert_allclose(g_b[s], g1, rtol=1e-5, atol=1e-6 * np.max(np.abs(g1)))


def test_unknown_and_skew_t_likelihoods_are_rejected():
    m = Model(10, 10)
    with pytest.raises(InvalidParameter):
        m.set_likelihood("st")
    with pytest.raises(InvalidParameter):
        m.set_likelihood("nonsense")
    m.set_likelihood("Student-T")  # aliases and case as profitParseLikefunc


def _mask_case(kind, w=100, h=90):
    yy, xx = np.mgrid[0:h, 0:w]
    if kind == "central":  # keeps psf/2 clear of every edge: no PSF padding
        return (((xx - 52) / 20.0) ** 2 + ((yy - 44) / 14.0) ** 2 < 1).astype(np.uint8)
    if kind == "edge":  # reaches the image edge: padding needed
        return ((xx < 30) & (yy > 50)).astype(np.uint8) | (((xx - 70) ** 2 + (yy - 30) ** 2) < 100).astype(np.uint8)
    raise ValueError(kind)


@pytest.mark.parametrize("kind,fs", [("central", 1), ("edge", 1), ("central", 2), ("edge", 3)])
def test_calculation_mask_matches_reference(kind, fs):
    """Model::set_mask with adjust_mask: drawing dimensions (PSF padding left
    out when the mask is clear of the edges), masked profiles, masked
    convolution and the final image &= mask, against the compiled reference."""
    psf = W.moffat_psf(15, 3.0, 2.5)
    mask = _mask_case(kind)
    out = []
    for M in (RefModel, Model):
        m = M(100, 90)
        m.set_magzero(30.0)  # a bright Sersic dominates the image
        m.set_psf(psf)
        m.set_finesampling(fs)
        m.set_return_finesampled(False)
        m.add_profile("sersic", xcen=52.3, ycen=44.1, re=6, nser=2.5, ang=30, axrat=0.6, convolve=True)
        m.add_profile("moffat", xcen=20.5, ycen=70.2, fwhm=3, con=2.5, convolve=False)
        m.add_profile("sky", bg=0.1)
        m.add_profile("psf", xcen=70.0, ycen=30.0, mag=16)
        m.set_mask(mask)
        out.append((m.drawing_dims(), m.evaluate()[0]))
    assert out[1][0] == out[0][0]
    assert out[1][1].shape == out[0][1].shape
    assert _rel(out[1][1], out[0][1]) <= IMG_TOL
    assert np.all(out[1][1][mask == 0] == 0)


def test_calculation_mask_without_adjustment_matches_reference():
    """adjust_mask = false: the mask is given at the drawing dimensions and
    used as it is (no dilation, no final mask)."""
    psf = W.gaussian_psf(11, 2.5)
    out = []
    for M in (RefModel, Model):
        m = M(60, 50)
        m.set_magzero(30.0)
        m.set_psf(psf)
        m.add_profile("sersic", xcen=30.2, ycen=25.7, re=5, nser=1.5, convolve=True)
        dw, dh = m.drawing_dims()
        yy, xx = np.mgrid[0:dh, 0:dw]
        m.set_mask(((xx - 35) ** 2 + (yy - 30) ** 2 < 300).astype(np.uint8), adjust=False)
        out.append(m.evaluate()[0])
    assert _rel(out[1], out[0]) <= IMG_TOL


def test_calculation_mask_errors():
    m = Model(40, 30)
    m.set_psf(W.gaussian_psf(7, 2.0))
    m.add_profile("sersic", xcen=20, ycen=15, re=3, convolve=True)
    m.set_mask(np.ones((10, 10), dtype=np.uint8))
    with pytest.raises(InvalidParameter):
        m.evaluate()  # Mask dimensions != model dimensions
    m.set_mask(np.ones((30, 40), dtype=np.uint8))
    m.evaluate()
    m.set_precision(PF_FP32)
    m.set_mask(np.ones((10, 10), dtype=np.uint8))
    with pytest.raises(InvalidParameter):
        m.evaluate()  # the FP32 form checks the same way


@pytest.mark.parametrize("kind", ["central", "edge"])
def test_calculation_mask_fft_equals_brute(kind):
    """The reference's FFT convolver is not compiled here (FFTW is absent); the
    masked FFT path must equal the masked brute-force path, which is pinned to
    the reference above."""
    psf = W.moffat_psf(15, 3.0, 2.5)
    out = []
    for conv in ("brute", "fft"):
        m = Model(100, 90)
        m.set_magzero(30.0)
        m.set_psf(psf)
        m.set_convolver(conv)
        m.add_profile("sersic", xcen=52.3, ycen=44.1, re=6, nser=2.5, ang=30, axrat=0.6, convolve=True)
        m.add_profile("sky", bg=0.1)
        m.set_mask(_mask_case(kind))
        out.append(m.evaluate()[0])
    assert _rel(out[1], out[0]) <= IMG_TOL


def test_dimensions_dry_run_and_threads():
    """Model::set_dimensions, set_dry_run (a zeroed drawing-size image, model.cpp:
    279-286) and set_omp_threads (accepted, no effect)."""
    m = Model(40, 30)
    m.set_psf(W.gaussian_psf(9, 2.0))
    m.add_profile("sersic", xcen=20, ycen=15, re=3, convolve=True)
    m.set_omp_threads(8)
    assert m.evaluate()[0].shape == (30, 40)
    m.set_dimensions(50, 20)
    img, _ = m.evaluate()
    assert img.shape == (20, 50) and img.max() > 0
    m.set_dry_run(True)
    img, off = m.evaluate()
    assert img.shape == (28, 58) and not img.any() and off == (0, 0)
    m.set_dimensions(0, 20)
    with pytest.raises(InvalidParameter):
        m.evaluate()


@pytest.mark.gpu
def test_convolver_benchmark_keeps_the_faster_convolver():
    """profitSetupData's benchmarked convolver choice (profitBenchmark +
    profitBenchmarkResultBest): both convolvers are timed, the faster one is
    kept, and the model then evaluates exactly as with that convolver set."""
    wl = W.single_sersic(seed_tag=21)
    m64 = W.configure(Model(wl["width"], wl["height"]), wl)
    ref, _ = m64.evaluate()
    image, sigma = W.make_data(wl, ref)
    # FP64 image (no data): the choice is one of the two, with both timed
    name, ms = m64.benchmark_convolvers(nbench=3)
    assert name in ("brute", "fft") and ms["brute"] > 0 and ms["fft"] > 0
    assert name == ("fft" if ms["fft"] < ms["brute"] else "brute")
    img, _ = m64.evaluate()
    assert _rel(img, ref) <= 1e-12
    # FP32 logL + gradient with data
    m32 = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), wl)
    m32.set_data(image, sigma)
    name, ms = m32.benchmark_convolvers(nbench=3)
    assert name in ("brute", "fft") and ms["brute"] > 0 and ms["fft"] > 0
    ll, g = m32.loglike_grad(wl["grad"])
    same = W.configure(Model(wl["width"], wl["height"], precision=PF_FP32), dict(wl, convolver=name))
    same.set_data(image, sigma)
    ll2, g2 = same.loglike_grad(wl["grad"])
    # (cells add to their pixel atomically, so two FP32 renders agree to
    # rounding, not bit for bit)
    assert ll == pytest.approx(ll2, rel=1e-7)
    np.testing.assert_allclose(g, g2, rtol=1e-5, atol=1e-6 * np.max(np.abs(g2)))
    with pytest.raises(InvalidParameter):
        m32.benchmark_convolvers(nbench=0)


def _fs_mask_model(mask, fs, precision=PF_FP32, conv="brute", adjust=True, retfine=False):
    """The calculation-mask case of the FP64 tests: a convolved bright Sersic,
    an unconvolved Moffat, sky and a psf point source (profile 3),
    finesampling fs."""
    m = Model(100, 90, precision=precision)
    m.set_magzero(30.0)
    m.set_psf(W.moffat_psf(15, 3.0, 2.5))
    m.set_convolver(conv)
    m.set_finesampling(fs)
    m.set_return_finesampled(retfine)
    m.add_profile("sersic", xcen=52.3, ycen=44.1, re=6, nser=2.5, ang=30, axrat=0.6, convolve=True)
    m.add_profile("moffat", xcen=20.5, ycen=70.2, fwhm=3, con=2.5, mag=19, convolve=False)
    m.add_profile("sky", bg=0.1)
    m.add_profile("psf", xcen=70.2, ycen=29.7, mag=16)
    if mask is not None:
        m.set_mask(mask, adjust)
    return m


@pytest.mark.parametrize("kind,fs,conv,retfine", [
    (None, 2, "brute", False), (None, 3, "fft", True), ("central", 1, "brute", False), ("edge", 1, "brute", False),
    ("central", 2, "fft", False), ("edge", 3, "brute", False), ("edge", 1, "fft", False)])
def test_fp32_masks_and_finesampling_match_fp64(kind, fs, conv, retfine):
    """The FP32 form with a calculation mask (masked profiles, masked
    convolution, image &= mask) and finesampling (summed down, or the fine
    image returned) against the plain FP64 form, to FP32 accuracy."""
    mask = None if kind is None else _mask_case(kind)
    m64 = _fs_mask_model(mask, fs, PF_FP64, conv, retfine=retfine)
    m32 = _fs_mask_model(mask, fs, PF_FP32, conv, retfine=retfine)
    assert m32.drawing_dims() == m64.drawing_dims()
    img64, off64 = m64.evaluate()
    img32, off32 = m32.evaluate()
    assert img32.shape == img64.shape and off32 == off64
    assert _rel(img32, img64) <= 1e-6
    if mask is not None:
        assert np.all(img32[mask == 0] == 0)


def test_fp32_mask_without_adjustment_matches_fp64():
    """adjust_mask = false: the drawing-size mask is used as given (masked
    profiles and convolution, no final mask)."""
    m64 = _fs_mask_model(None, 1, PF_FP64)
    dw, dh = m64.drawing_dims()
    yy, xx = np.mgrid[0:dh, 0:dw]
    mask = (((xx - 60) / 30.0) ** 2 + ((yy - 50) / 25.0) ** 2 < 1).astype(np.uint8)
    imgs = []
    for prec in (PF_FP64, PF_FP32):
        m = _fs_mask_model(None, 1, prec)
        m.set_mask(mask, adjust=False)
        imgs.append(m.evaluate()[0])
    assert _rel(imgs[1], imgs[0]) <= 1e-6


@pytest.mark.parametrize("kind,fs,conv", [("central", 1, "brute"), ("edge", 2, "brute"), ("edge", 1, "fft"),
                                          (None, 2, "fft")])
def test_fp32_adjoint_with_mask_and_finesampling_matches_fd64(kind, fs, conv):
    """d logL / d(parameters) through masked rendering, masked convolution,
    the sum-down of the finesampled image and image &= mask, and the centre
    and magnitude of a psf point source (its area-overlap stamp), against FP64
    central differences of the plain form (store and recompute adjoints, one
    proposal and a batch)."""
    from profit_b200._capi import PF_ADJOINT_RECOMPUTE, PF_ADJOINT_STORE
    mask = None if kind is None else _mask_case(kind)
    truth = _fs_mask_model(mask, fs, PF_FP64, conv)
    img, _ = truth.evaluate()
    rng = np.random.Generator(np.random.PCG64(31))
    sigma = 1.0 + 0.1 * np.sqrt(np.abs(img))
    image = img + rng.normal(0.0, 1.0, img.shape) * sigma
    refs = [(0, "xcen"), (0, "ycen"), (0, "mag"), (0, "re"), (0, "nser"), (0, "ang"), (0, "axrat"),
            (1, "xcen"), (1, "ycen"), (1, "mag"), (3, "xcen"), (3, "ycen"), (3, "mag")]
    prop = [52.6, 43.8, 15.05, 6.2, 2.45, 31.0, 0.62, 20.3, 70.4, 19.03, 70.35, 29.6, 16.03]
    m = _fs_mask_model(mask, fs, PF_FP64, conv)
    m.set_data(image, sigma)
    m.set_parameters(refs, prop)
    ll64 = m.loglike()
    _, g6 = m.loglike_grad_fd(refs, rel_step=1e-6)
    _, g5 = m.loglike_grad_fd(refs, rel_step=1e-5)
    scale = np.max(np.abs(g6))
    spread = 2 * np.abs(g6 - g5) / scale
    m.set_precision(PF_FP32)
    for mode in (PF_ADJOINT_STORE, PF_ADJOINT_RECOMPUTE):
        m.set_adjoint_mode(mode)
        for _ in range(2):  # eager, then graph replay
            ll32, g = m.loglike_grad(refs)
            assert ll32 == pytest.approx(ll64, rel=1e-5)
            err = np.minimum(np.abs(g - g6), np.abs(g - g5)) / scale
            assert np.all(err <= np.maximum(1e-5, spread)), (mode, list(zip(refs, g6, g5, g)))
    m.set_adjoint_mode(PF_ADJOINT_STORE)
    vals = np.array([prop, [v * (1 + 1e-3) for v in prop]])
    ll_b, g_b = m.loglike_grad_batch(refs, vals)
    for s in range(2):
        m.set_parameters(refs, vals[s])
        l1, g1 = m.loglike_grad(refs)
        # (a batch of two may run other autotuned convolution tiles than one
        # proposal: FP32 sums in another order)
        assert ll_b[s] == pytest.approx(l1, rel=1e-6)
        np.testing.assert_allclose(g_b[s], g1, rtol=1e-5, atol=1e-6 * np.max(np.abs(g1)))


@pytest.mark.parametrize("conv", ["brute", "brute-old", "null"])
@pytest.mark.parametrize("crop", [True, False])
def test_convolvers_and_crop_match_reference(conv, crop):
    """"brute-old" (BruteForceConvolver, convolve.cpp:101-156: one running
    sum per output pixel with edge clipping) and "brute"
    (AssociativeBruteForceConvolver, row dot products) sum in different
    orders; both agree with the compiled reference's own convolver of that
    name to 1e-12, with and without a calculation mask.  crop = false
    (model.cpp:307-322) returns the cropped image for these convolvers, since
    they add no padding of their own; the offset stays (0, 0)."""
    psf = W.moffat_psf(15, 3.0, 2.5)
    mask = _mask_case("edge")
    for use_mask in (False, True):
        out = []
        for M in (RefModel, Model):
            m = M(100, 90)
            m.set_magzero(30.0)
            m.set_psf(psf)
            m.set_convolver(conv)
            m.set_crop(crop)
            m.add_profile("sersic", xcen=52.3, ycen=44.1, re=6, nser=2.5, ang=30, axrat=0.6, convolve=True)
            m.add_profile("moffat", xcen=20.5, ycen=70.2, fwhm=3, con=2.5, convolve=False)
            m.add_profile("sky", bg=0.1)
            if use_mask:
                m.set_mask(mask)
            out.append(m.evaluate())
        (ref, ref_off), (got, got_off) = out
        assert got.shape == ref.shape == (90, 100)
        assert got_off == ref_off == (0, 0)
        assert _rel(got, ref) <= IMG_TOL


def test_crop_false_with_fft_is_refused():
    m = Model(40, 30)
    m.set_psf(W.gaussian_psf(9, 2.0))
    m.set_convolver("fft")
    m.set_crop(False)
    m.add_profile("sersic", xcen=20, ycen=15, re=3, convolve=True)
    with pytest.raises(InvalidParameter, match="crop = false"):
        m.evaluate()
    m.set_crop(True)
    assert m.evaluate()[0].shape == (30, 40)
