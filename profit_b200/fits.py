"""FITS input for fits of real data, and ProFit's default data set-up.

ProFit's vignettes read a galaxy cut-out as five FITS images with Rfits (image,
sigma map, segmentation map, mask and PSF: inst/extdata/KiDS/G*{fitim,sigma,
segim,mskim,psfim}.fits) and pass them to profitSetupData
(R/profitSetupData.R:151-340). This module reads and writes FITS images
(primary HDU or the first IMAGE extension holding data; BITPIX 8, 16, 32, 64,
-32 and -64; BSCALE/BZERO applied) and restates profitSetupData's defaults
for the region the likelihood covers.

Arrays are returned as [NAXIS2, NAXIS1] float64, i.e. [height, width] with x
(the first FITS axis) fastest, which is the layout profit_b200.Model takes.
"""
from __future__ import annotations

import math
import os
from typing import Dict, Optional, Tuple

import numpy as np

BLOCK = 2880
CARD = 80
_DTYPES = {8: ">u1", 16: ">i2", 32: ">i4", 64: ">i8", -32: ">f4", -64: ">f8"}


class FitsError(ValueError):
    pass


def _parse_value(text: str):
    """Value field of a card (after '= '), comment stripped."""
    t = text.strip()
    if t.startswith("'"):
        # quoted string: '' is an escaped quote; trailing blanks are not significant
        out, i = [], 1
        while i < len(t):
            if t[i] == "'":
                if i + 1 < len(t) and t[i + 1] == "'":
                    out.append("'")
                    i += 2
                    continue
                break
            out.append(t[i])
            i += 1
        return "".join(out).rstrip()
    if "/" in t:
        t = t[:t.index("/")].strip()
    if t == "T":
        return True
    if t == "F":
        return False
    if t == "":
        return None
    try:
        return int(t)
    except ValueError:
        pass
    try:
        return float(t.replace("D", "E").replace("d", "e"))
    except ValueError:
        return t


def _read_header(f) -> Tuple[Dict[str, object], bool]:
    """Cards up to END (keyword -> value; COMMENT/HISTORY dropped). Returns
    (header, found); found is False at end of file."""
    header: Dict[str, object] = {}
    while True:
        block = f.read(BLOCK)
        if not block:
            if header:
                raise FitsError("header without END")
            return header, False
        if len(block) != BLOCK:
            raise FitsError("truncated header block")
        for k in range(0, BLOCK, CARD):
            card = block[k:k + CARD].decode("ascii", errors="replace")
            key = card[:8].strip()
            if key == "END":
                return header, True
            if key in ("", "COMMENT", "HISTORY") or card[8:10] != "= ":
                continue
            header[key] = _parse_value(card[10:])


def _data_bytes(h: Dict[str, object]) -> int:
    bitpix = int(h.get("BITPIX", 8))
    naxis = int(h.get("NAXIS", 0))
    if naxis == 0:
        n = 0
    else:
        n = 1
        for i in range(1, naxis + 1):
            n *= int(h[f"NAXIS{i}"])
    n = abs(bitpix) // 8 * int(h.get("GCOUNT", 1)) * (int(h.get("PCOUNT", 0)) + n)
    return n


def read_fits(path: str) -> Tuple[np.ndarray, Dict[str, object]]:
    """The first image with data in a FITS file: (array [NAXIS2, NAXIS1] or
    with more axes [..., NAXIS2, NAXIS1] squeezed of length-1 axes, header)."""
    with open(path, "rb") as f:
        first = True
        while True:
            h, found = _read_header(f)
            if not found:
                raise FitsError(f"{path}: no image HDU with data")
            if first and h.get("SIMPLE") is not True:
                raise FitsError(f"{path}: not a FITS file (SIMPLE != T)")
            nbytes = _data_bytes(h)
            is_image = first or h.get("XTENSION") == "IMAGE"
            first = False
            if is_image and int(h.get("NAXIS", 0)) >= 2 and nbytes > 0:
                bitpix = int(h["BITPIX"])
                if bitpix not in _DTYPES:
                    raise FitsError(f"{path}: unsupported BITPIX {bitpix}")
                naxis = int(h["NAXIS"])
                shape = tuple(int(h[f"NAXIS{i}"]) for i in range(naxis, 0, -1))
                count = int(np.prod(shape))
                raw = f.read(count * abs(bitpix) // 8)
                if len(raw) != count * abs(bitpix) // 8:
                    raise FitsError(f"{path}: truncated data")
                a = np.frombuffer(raw, dtype=_DTYPES[bitpix]).astype(np.float64).reshape(shape)
                scale, zero = float(h.get("BSCALE", 1.0)), float(h.get("BZERO", 0.0))
                if scale != 1.0 or zero != 0.0:
                    a = zero + scale * a
                if "BLANK" in h and bitpix > 0:  # undefined integer pixels
                    raw_int = np.frombuffer(raw, dtype=_DTYPES[bitpix]).reshape(shape)
                    a = np.where(raw_int == int(h["BLANK"]), np.nan, a)
                while a.ndim > 2 and a.shape[0] == 1:
                    a = a[0]
                return np.ascontiguousarray(a), h
            # skip this HDU's data (padded to whole blocks)
            f.seek(int(math.ceil(nbytes / BLOCK)) * BLOCK, os.SEEK_CUR)


def _card(key: str, value, comment: str = "") -> bytes:
    if isinstance(value, bool):
        v = f"{'T' if value else 'F':>20}"
    elif isinstance(value, (int, np.integer)):
        v = f"{int(value):>20d}"
    elif isinstance(value, (float, np.floating)):
        v = f"{float(value):>20.17G}"
    else:
        v = "'" + str(value).replace("'", "''").ljust(8) + "'"
    text = f"{key:<8}= {v}"
    if comment:
        text += f" / {comment}"
    return text[:CARD].ljust(CARD).encode("ascii")


def write_fits(path: str, image: np.ndarray, bitpix: int = -64, header: Optional[Dict[str, object]] = None,
               bscale: float = 1.0, bzero: float = 0.0) -> None:
    """A single-HDU FITS image of a [NAXIS2, NAXIS1] array. Integer BITPIX
    stores round((image - bzero) / bscale)."""
    if bitpix not in _DTYPES:
        raise FitsError(f"unsupported BITPIX {bitpix}")
    a = np.asarray(image, dtype=np.float64)
    if a.ndim != 2:
        raise FitsError("write_fits takes a 2-D array")
    cards = [_card("SIMPLE", True, "conforms to FITS standard"), _card("BITPIX", bitpix), _card("NAXIS", 2),
             _card("NAXIS1", a.shape[1]), _card("NAXIS2", a.shape[0])]
    if bitpix > 0 or bscale != 1.0 or bzero != 0.0:
        cards += [_card("BSCALE", float(bscale)), _card("BZERO", float(bzero))]
    for k, v in (header or {}).items():
        cards.append(_card(k, v))
    cards.append(b"END".ljust(CARD))
    head = b"".join(cards)
    head += b" " * ((-len(head)) % BLOCK)
    raw = (a - bzero) / bscale
    if bitpix > 0:
        raw = np.rint(raw)
    data = raw.astype(_DTYPES[bitpix]).tobytes()
    data += b"\0" * ((-len(data)) % BLOCK)
    with open(path, "wb") as f:
        f.write(head)
        f.write(data)


def read_cutout(prefix: str) -> Dict[str, Optional[np.ndarray]]:
    """The five images of a ProFit example cut-out, <prefix>{fitim, sigma,
    segim, mskim, psfim}.fits, as image, sigma, segim, mask, psf (None where a
    file is absent)."""
    out: Dict[str, Optional[np.ndarray]] = {}
    for key, suffix in (("image", "fitim"), ("sigma", "sigma"), ("segim", "segim"), ("mask", "mskim"),
                        ("psf", "psfim")):
        p = f"{prefix}{suffix}.fits"
        out[key] = read_fits(p)[0] if os.path.exists(p) else None
    return out


def setup_region(image: np.ndarray, sigma: Optional[np.ndarray] = None, segim: Optional[np.ndarray] = None,
                 mask: Optional[np.ndarray] = None) -> Tuple[np.ndarray, np.ndarray]:
    """profitSetupData's defaults (R/profitSetupData.R:171-232): sigma =
    sqrt(|image|) when absent; the region the likelihood covers is the
    segment of the central pixel (R's segim[ceiling(W/2), ceiling(H/2)]) minus
    the masked pixels (mask > 0). Returns (sigma, region as uint8). The same
    region, as the calculation mask, is what ProFit adjusts into calcregion
    (Model.set_mask with adjust)."""
    image = np.asarray(image, dtype=np.float64)
    h, w = image.shape
    if sigma is None:
        sigma = np.sqrt(np.abs(image))
    if segim is None:
        segim = np.ones_like(image)
    if mask is None:
        mask = np.zeros_like(image)
    keep = segim[int(math.ceil(h / 2)) - 1, int(math.ceil(w / 2)) - 1]
    region = ((segim == keep) & (mask <= 0)).astype(np.uint8)
    return np.asarray(sigma, dtype=np.float64), region
