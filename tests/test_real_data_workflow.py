"""A fit's data path end to end on the GPU: a cut-out written as the five FITS
images of ProFit's examples (image, sigma, segmentation, mask, PSF), read
back, set up with profitSetupData's region rule, and evaluated with the region
as both the likelihood region and the calculation mask (ProFit's calcregion),
FP32 logL and adjoint gradient against the plain FP64 form and FD."""
import numpy as np
import pytest

from profit_b200 import PF_FP32, PF_FP64, Model
from profit_b200 import workloads as W
from profit_b200.fits import read_cutout, setup_region, write_fits

pytestmark = pytest.mark.gpu


def _write_cutout(prefix, w=120, h=96):
    """A bright Sersic galaxy with a neighbour, a segmentation map that
    separates them, a masked star and a Moffat PSF."""
    truth = Model(w, h)
    truth.set_magzero(30.0)
    psf = W.moffat_psf(21, 3.0, 2.5)
    truth.set_psf(psf)
    truth.add_profile("sersic", xcen=60.3, ycen=48.2, mag=17.0, re=7.0, nser=2.2, ang=40, axrat=0.7, convolve=True)
    truth.add_profile("sersic", xcen=18.0, ycen=80.0, mag=19.0, re=3.0, nser=1.0, convolve=True)
    img, _ = truth.evaluate()
    rng = np.random.Generator(np.random.PCG64(12))
    sigma = 1.0 + 0.05 * np.sqrt(np.abs(img))
    image = img + rng.normal(size=img.shape) * sigma
    yy, xx = np.mgrid[0:h, 0:w]
    seg = np.where(((xx - 60) / 40.0) ** 2 + ((yy - 48) / 30.0) ** 2 < 1, 3, 0)
    seg = np.where(((xx - 18) ** 2 + (yy - 80) ** 2) < 100, 5, seg)
    mask = (((xx - 90) ** 2 + (yy - 30) ** 2) < 16).astype(float)
    write_fits(prefix + "fitim.fits", image, bitpix=-32)
    write_fits(prefix + "sigma.fits", sigma, bitpix=-32)
    write_fits(prefix + "segim.fits", seg, bitpix=16)
    write_fits(prefix + "mskim.fits", mask, bitpix=8)
    write_fits(prefix + "psfim.fits", psf, bitpix=-64)


def test_fits_cutout_fit_path(tmp_path):
    prefix = str(tmp_path / "G1")
    _write_cutout(prefix)
    c = read_cutout(prefix)
    sigma, region = setup_region(c["image"], c["sigma"], c["segim"], c["mask"])
    assert region.sum() > 0 and not region[30, 90]  # the masked star is out
    h, w = c["image"].shape
    refs = [(0, "xcen"), (0, "ycen"), (0, "mag"), (0, "re"), (0, "nser"), (0, "ang"), (0, "axrat")]
    prop = [60.5, 48.0, 17.02, 7.1, 2.15, 41.0, 0.71]

    def model(prec):
        m = Model(w, h, precision=prec)
        m.set_magzero(30.0)
        m.set_psf(c["psf"])
        m.add_profile("sersic", xcen=60.3, ycen=48.2, mag=17.0, re=7.0, nser=2.2, ang=40, axrat=0.7, convolve=True)
        m.set_data(c["image"], sigma, region)
        m.set_mask(region)  # ProFit's calcregion: the region, adjusted
        m.set_parameters(refs, prop)
        return m

    m64 = model(PF_FP64)
    ll64 = m64.loglike()
    _, g6 = m64.loglike_grad_fd(refs, rel_step=1e-6)
    _, g5 = m64.loglike_grad_fd(refs, rel_step=1e-5)
    m32 = model(PF_FP32)
    ll32, g = m32.loglike_grad(refs)
    assert ll32 == pytest.approx(ll64, rel=1e-5)
    scale = np.max(np.abs(g6))
    err = np.minimum(np.abs(g - g6), np.abs(g - g5)) / scale
    assert np.all(err <= np.maximum(1e-5, 2 * np.abs(g6 - g5) / scale)), list(zip(refs, g6, g5, g))
