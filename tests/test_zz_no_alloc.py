"""pf_loglike_norm_noalloc: the log-likelihood of device-resident images with
its scratch in a static device array.  Compared with pf_model_loglike on two
calls in a row, the second of which reuses the array the first one left
behind.  Kept in its own file, collected last, so it also runs after every
other test has used the library in the same process."""
import numpy as np
import pytest

from profit_b200 import Model
from profit_b200 import workloads as W
from profit_b200._capi import PF_E_CAPACITY, PF_LOGLIKE_NOALLOC_MAX_BATCH, PF_OK, check, lib

pytestmark = pytest.mark.gpu


def _proposal(wl, seed, image, sigma, region=None):
    """(model image, pf_model_loglike) of one perturbed proposal."""
    p = W.perturbed(wl, seed)
    m = W.configure(Model(p["width"], p["height"]), p)
    m.set_data(image, sigma, region)
    ll = m.loglike()
    img, _ = m.evaluate()
    return img, ll


def test_static_scratch_loglike_matches_model_loglike():
    import torch

    wl = W.bulge_disk_ps()
    truth, _ = W.configure(Model(wl["width"], wl["height"]), wl).evaluate()
    image, sigma = W.make_data(wl, truth)
    region = (np.random.Generator(np.random.PCG64(17)).uniform(size=image.shape) < 0.8).astype(np.uint8)

    img_a, ll_a = _proposal(wl, 1, image, sigma)
    img_b, ll_b = _proposal(wl, 2, image, sigma)
    img_c, ll_c = _proposal(wl, 3, image, sigma, region)
    npix = image.size

    dev = torch.device("cuda:0")
    d_models = torch.tensor(np.stack([img_a, img_b, img_a]), dtype=torch.float64, device=dev)
    d_c = torch.tensor(img_c, dtype=torch.float64, device=dev)
    d_data = torch.tensor(image, dtype=torch.float64, device=dev)
    d_sigma = torch.tensor(sigma, dtype=torch.float64, device=dev)
    d_region = torch.tensor(region, dtype=torch.uint8, device=dev)
    d_ll = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    L = lib()

    # call 1: three images against the same data, all pixels.  pf_model_loglike
    # renders its own image, which can differ from the one evaluate() returned
    # in the last bit (subsampled pixels are summed atomically), hence the
    # tolerance; the same image twice gives the same sum exactly.
    check(L.pf_loglike_norm_noalloc(d_models.data_ptr(), d_data.data_ptr(), d_sigma.data_ptr(), None, npix, 3,
                                    d_ll.data_ptr(), stream.cuda_stream))
    stream.synchronize()
    got = d_ll.cpu().numpy()
    assert got[0] == pytest.approx(ll_a, rel=1e-12)
    assert got[1] == pytest.approx(ll_b, rel=1e-12)
    assert got[2] == got[0]

    # call 2: one proposal with a region mask, on the scratch call 1 left;
    # the device's free memory must not move.
    d_ll.fill_(float("nan"))
    stream.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    check(L.pf_loglike_norm_noalloc(d_c.data_ptr(), d_data.data_ptr(), d_sigma.data_ptr(), d_region.data_ptr(),
                                    npix, 1, d_ll.data_ptr(), stream.cuda_stream))
    stream.synchronize()
    free_after = torch.cuda.mem_get_info(dev)[0]
    got = d_ll.cpu().numpy()
    assert got[0] == pytest.approx(ll_c, rel=1e-12)
    assert np.isnan(got[1:]).all()  # only `batch` results are written
    assert free_after == free_before


def test_static_scratch_loglike_rejects_batches_beyond_its_size():
    import torch

    dev = torch.device("cuda:0")
    npix = 64
    n = PF_LOGLIKE_NOALLOC_MAX_BATCH + 1
    # buffers large enough for the refused batch, so nothing could read past them
    d_models = torch.zeros((n, npix), dtype=torch.float64, device=dev)
    d_data = torch.zeros(npix, dtype=torch.float64, device=dev)
    d_sigma = torch.ones(npix, dtype=torch.float64, device=dev)
    d_ll = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    L = lib()
    st = L.pf_loglike_norm_noalloc(d_models.data_ptr(), d_data.data_ptr(), d_sigma.data_ptr(), None, npix, n,
                                   d_ll.data_ptr(), stream.cuda_stream)
    assert st == PF_E_CAPACITY
    assert b"PF_LOGLIKE_NOALLOC_MAX_BATCH" in L.pf_last_error()
    stream.synchronize()
    assert torch.isnan(d_ll).all()
    # the largest batch it takes: zero residuals give -n/2 log(2 pi) per image
    st = L.pf_loglike_norm_noalloc(d_models.data_ptr(), d_data.data_ptr(), d_sigma.data_ptr(), None, npix, n - 1,
                                   d_ll.data_ptr(), stream.cuda_stream)
    assert st == PF_OK
    stream.synchronize()
    got = d_ll.cpu().numpy()
    assert np.allclose(got[: n - 1], -npix * 0.5 * np.log(2 * np.pi), rtol=1e-14)
    assert np.isnan(got[n - 1])


@pytest.mark.parametrize("w,h", [(100, 100), (37, 23), (400, 380)])
def test_static_scratch_loglike_equals_model_loglike_bit_for_bit(w, h):
    """Images below 151,552 pixels reduce over fewer than 296 blocks in
    pf_model_loglike; the static-scratch call must use the same grid and give
    the same logL to the last bit.  A rough profile (no subsampling, so no
    atomically summed cells) and sky make the FP64 model image reproducible,
    so both calls see the same image."""
    import torch

    psf = W.gaussian_psf(9, 2.0)
    m = Model(w, h)
    m.set_magzero(25.0)
    m.set_psf(psf)
    m.add_profile("sersic", xcen=w * 0.45, ycen=h * 0.55, mag=15.0, re=w * 0.1, nser=2.0, ang=30.0, axrat=0.7,
                  rough=True, convolve=True)
    m.add_profile("sky", bg=0.5)
    img, _ = m.evaluate()
    image, sigma = W.make_data(dict(sigma_range=(0.5, 2.0), seed_tag=71), img)
    m.set_data(image, sigma)
    ll = m.loglike()
    again, _ = m.evaluate()
    assert np.array_equal(again, img)

    dev = torch.device("cuda:0")
    d_model = torch.tensor(np.stack([img, img]), dtype=torch.float64, device=dev)
    d_data = torch.tensor(image, dtype=torch.float64, device=dev)
    d_sigma = torch.tensor(sigma, dtype=torch.float64, device=dev)
    d_ll = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    L = lib()
    for _ in range(2):  # the second call runs on the scratch the first left
        d_ll.fill_(float("nan"))
        check(L.pf_loglike_norm_noalloc(d_model.data_ptr(), d_data.data_ptr(), d_sigma.data_ptr(), None, img.size,
                                        2, d_ll.data_ptr(), stream.cuda_stream))
        stream.synchronize()
        got = d_ll.cpu().numpy()
        assert got[0] == ll and got[1] == ll
