"""FITS input (profit_b200.fits) and profitSetupData's region defaults, on the
CPU: round trips for every BITPIX, a hand-assembled known-answer file, and
(where the ProFit tree is present) the reference's own KiDS example cut-out."""
import os
import struct

import numpy as np
import pytest

from oracle.refpath import reference_root
from profit_b200.fits import FitsError, read_cutout, read_fits, setup_region, write_fits

KIDS = os.path.join(reference_root(), "inst", "extdata", "KiDS", "G266035")


@pytest.mark.parametrize("bitpix", [-64, -32, 8, 16, 32, 64])
def test_round_trip(tmp_path, bitpix):
    rng = np.random.default_rng(1)
    a = rng.uniform(0, 200, size=(7, 11))
    kw = {}
    if bitpix > 0:
        a = np.rint(a)
        if bitpix == 16:
            kw = dict(bscale=0.5, bzero=10.0)  # stored ints (a - 10) / 0.5
    p = str(tmp_path / "x.fits")
    write_fits(p, a, bitpix=bitpix, header={"OBJECT": "test's", "GAIN": 2.5}, **kw)
    assert os.path.getsize(p) % 2880 == 0
    b, h = read_fits(p)
    assert b.shape == (7, 11) and h["NAXIS1"] == 11 and h["NAXIS2"] == 7
    assert h["OBJECT"] == "test's" and h["GAIN"] == 2.5
    tol = 1e-6 * np.abs(a).max() if bitpix == -32 else 0
    np.testing.assert_allclose(b, a, atol=tol, rtol=0)


def test_known_answer_file(tmp_path):
    """A file assembled card by card: 3x2 big-endian int16 with BZERO 32768
    (the unsigned convention), a blank pixel, then an IMAGE extension that the
    reader must not reach."""
    def card(s):
        return s.ljust(80).encode()
    head = b"".join(card(c) for c in [
        "SIMPLE  =                    T", "BITPIX  =                   16", "NAXIS   =                    2",
        "NAXIS1  =                    3", "NAXIS2  =                    2", "BZERO   =              32768.0",
        "BLANK   =                -1000", "TELESCOP= 'VST     '           / comment", "END"])
    head += b" " * (2880 - len(head))
    vals = [-32768, 0, 32767, 5, -1000, 7]
    data = struct.pack(">6h", *vals)
    data += b"\0" * (2880 - len(data))
    p = tmp_path / "k.fits"
    p.write_bytes(head + data)
    a, h = read_fits(str(p))
    assert h["TELESCOP"] == "VST"
    assert a.shape == (2, 3)
    np.testing.assert_array_equal(a[0], [0, 32768, 65535])
    assert a[1, 0] == 32773 and np.isnan(a[1, 1]) and a[1, 2] == 32775


def test_image_extension_after_empty_primary(tmp_path):
    def card(s):
        return s.ljust(80).encode()
    def block(cards):
        b = b"".join(card(c) for c in cards)
        return b + b" " * ((-len(b)) % 2880)
    prim = block(["SIMPLE  =                    T", "BITPIX  =                    8", "NAXIS   =                    0",
                  "EXTEND  =                    T", "END"])
    ext = block(["XTENSION= 'IMAGE   '", "BITPIX  =                  -64", "NAXIS   =                    2",
                 "NAXIS1  =                    2", "NAXIS2  =                    2", "PCOUNT  =                    0",
                 "GCOUNT  =                    1", "END"])
    data = struct.pack(">4d", 1.5, -2.0, 3.25, 1e300)
    data += b"\0" * ((-len(data)) % 2880)
    p = tmp_path / "e.fits"
    p.write_bytes(prim + ext + data)
    a, _ = read_fits(str(p))
    np.testing.assert_array_equal(a, [[1.5, -2.0], [3.25, 1e300]])


def test_not_fits_is_rejected(tmp_path):
    p = tmp_path / "n.fits"
    p.write_bytes(b"hello".ljust(2880))
    with pytest.raises(FitsError):
        read_fits(str(p))


def test_setup_region_follows_profitsetupdata():
    """region = segment of the central pixel (R: segim[ceiling(W/2),
    ceiling(H/2)], 1-based, x first) and not masked; sigma = sqrt|image|."""
    img = np.arange(4 * 5, dtype=float).reshape(4, 5) - 3.0  # H = 4, W = 5
    seg = np.zeros((4, 5))
    seg[1:3, 1:4] = 7      # centre pixel (x = 3, y = 2 in R) is at [1, 2]
    seg[0, 0] = 7
    mask = np.zeros((4, 5))
    mask[2, 3] = 1
    sigma, region = setup_region(img, segim=seg, mask=mask)
    np.testing.assert_allclose(sigma, np.sqrt(np.abs(img)))
    expect = (seg == 7) & (mask <= 0)
    np.testing.assert_array_equal(region, expect.astype(np.uint8))
    _, all_in = setup_region(img)
    assert all_in.all()


@pytest.mark.skipif(not os.path.exists(KIDS + "fitim.fits"), reason="ProFit example data not present")
def test_reference_kids_cutout():
    """The reference's KiDS example cut-out reads with consistent shapes: a
    209 x 155 image (BITPIX -32), its sigma, segmentation and mask maps, and a
    PSF whose central pixel is its maximum."""
    c = read_cutout(KIDS)
    assert c["image"].shape == (155, 209)
    for k in ("sigma", "segim", "mask"):
        assert c[k].shape == c["image"].shape
    assert np.all(np.isfinite(c["image"])) and np.all(c["sigma"] > 0)
    psf = c["psf"]
    assert psf.ndim == 2 and psf.shape[0] % 2 == 1 and psf.shape[1] % 2 == 1
    assert psf[psf.shape[0] // 2, psf.shape[1] // 2] == psf.max()
    sigma, region = setup_region(c["image"], c["sigma"], c["segim"], c["mask"])
    assert 0 < region.sum() < region.size
