"""Seeded synthetic inputs with the shapes of ProFit's benchmark configurations.

No public dataset is involved: every image, PSF, sigma map and parameter set
comes from numpy's PCG64 generator with a fixed seed per configuration.

  single_sersic   100x100 Sersic + 25x25 Gaussian PSF (FWHM 3), brute force,
                  sigma = 1 (the plain CPU-runnable case)
  bulge_disk_ps   400x400 Sersic bulge + exponential disk + unconvolved Moffat
                  point source, 51x51 Moffat PSF, sigma ~ U[0.5, 2]

A workload is a plain dict:
  width, height, magzero, psf (2-D array), convolver,
  profiles: list of (name, {param: value}),
  grad: list of (profile index, parameter name) for gradients,
  image, sigma: data arrays (filled by make_data()).
"""
from __future__ import annotations

import math
from typing import Dict, List, Tuple

import numpy as np

SEED = 20261203


def gaussian_psf(size: int, fwhm: float) -> np.ndarray:
    """Unit-sum Gaussian sampled at pixel centres, centred on the middle pixel."""
    s = fwhm / (2.0 * math.sqrt(2.0 * math.log(2.0)))
    c = (size - 1) / 2.0
    y, x = np.mgrid[0:size, 0:size]
    p = np.exp(-((x - c) ** 2 + (y - c) ** 2) / (2 * s * s))
    return p / p.sum()


def moffat_psf(size: int, fwhm: float, con: float) -> np.ndarray:
    """Unit-sum circular Moffat (1 + (r/rs)^2)^-con with FWHM `fwhm`."""
    rs = fwhm / (2.0 * math.sqrt(2.0 ** (1.0 / con) - 1.0))
    c = (size - 1) / 2.0
    y, x = np.mgrid[0:size, 0:size]
    r2 = ((x - c) ** 2 + (y - c) ** 2) / (rs * rs)
    p = (1.0 + r2) ** (-con)
    return p / p.sum()


def _rng(tag: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64([SEED, tag]))


def single_sersic(seed_tag: int = 1, width: int = 100, height: int = 100, psf_size: int = 25) -> Dict:
    r = _rng(seed_tag)
    prof = dict(xcen=r.uniform(45, 55) * width / 100.0, ycen=r.uniform(45, 55) * height / 100.0, mag=15.0,
                re=r.uniform(5, 12), nser=r.uniform(1, 4), ang=r.uniform(0, 180), axrat=r.uniform(0.4, 1.0),
                box=0.0, convolve=True)
    return dict(name="single_sersic", width=width, height=height, magzero=0.0,
                psf=gaussian_psf(psf_size, 3.0), convolver="brute",
                profiles=[("sersic", prof)],
                grad=[(0, k) for k in ("xcen", "ycen", "mag", "re", "nser", "ang", "axrat", "box")],
                sigma_range=(1.0, 1.0), seed_tag=seed_tag)


def bulge_disk_ps(seed_tag: int = 2, width: int = 400, height: int = 400, psf_size: int = 51,
                  magzero: float = 30.0) -> Dict:
    """Bulge + disk + point source.  Magnitudes (not fixed by the configuration)
    are chosen so the bulge peak is tens of sigma above the noise."""
    r = _rng(seed_tag)
    cx, cy = width / 2.0 + r.uniform(-5, 5), height / 2.0 + r.uniform(-5, 5)
    bulge = dict(xcen=cx + r.uniform(-0.5, 0.5), ycen=cy + r.uniform(-0.5, 0.5), mag=r.uniform(19.5, 20.5),
                 re=r.uniform(2, 10), nser=float(np.exp(r.uniform(np.log(2), np.log(8)))), ang=r.uniform(0, 180),
                 axrat=r.uniform(0.5, 1.0), box=0.0, convolve=True)
    disk = dict(xcen=cx + r.uniform(-0.5, 0.5), ycen=cy + r.uniform(-0.5, 0.5), mag=r.uniform(18.5, 19.5),
                re=r.uniform(10, 40), nser=1.0, ang=r.uniform(0, 180), axrat=r.uniform(0.2, 1.0), box=0.0,
                convolve=True)
    ps = dict(xcen=r.uniform(0.25, 0.75) * width, ycen=r.uniform(0.25, 0.75) * height, mag=r.uniform(20.5, 21.5),
              fwhm=3.0, con=2.5, convolve=False)
    grad = [(0, k) for k in ("xcen", "ycen", "mag", "re", "nser", "ang", "axrat", "box")]
    grad += [(1, k) for k in ("xcen", "ycen", "mag", "re", "ang", "axrat")]
    grad += [(2, k) for k in ("xcen", "ycen", "mag")]
    return dict(name="bulge_disk_ps", width=width, height=height, magzero=magzero,
                psf=moffat_psf(psf_size, 3.0, 2.5), convolver="brute",
                profiles=[("sersic", bulge), ("sersic", disk), ("moffat", ps)], grad=grad,
                sigma_range=(0.5, 2.0), seed_tag=seed_tag)


def sampler_batch(n: int = 4096, seed_tag: int = 3) -> Tuple[Dict, np.ndarray]:
    """The single-Sersic model at 200x200 with a 31x31 Gaussian PSF and n
    sampler proposals params = init + N(0, 0.05 |init|) (redrawn until valid).
    Returns (workload, values[n, 8]) for the 8 Sersic parameters."""
    wl = single_sersic(seed_tag=seed_tag, width=200, height=200, psf_size=31)
    refs = wl["grad"]
    init = np.array([wl["profiles"][i][1][k] for (i, k) in refs])
    r = np.random.Generator(np.random.PCG64([SEED, 91, seed_tag]))
    vals = init + r.normal(size=(n, len(refs))) * 0.05 * np.abs(init)
    for j, (_, k) in enumerate(refs):
        lo = {"axrat": 0.05, "re": 1e-3, "nser": 0.3}.get(k)
        hi = {"axrat": 1.0}.get(k)
        for _ in range(100):
            bad = np.zeros(n, dtype=bool)
            if lo is not None:
                bad |= vals[:, j] <= lo
            if hi is not None:
                bad |= vals[:, j] > hi
            if not bad.any():
                break
            vals[bad, j] = init[j] + r.normal(size=bad.sum()) * 0.05 * abs(init[j])
    return wl, vals


def large_field(n_profiles: int = 200, width: int = 2000, height: int = 2000, psf_size: int = 101,
                seed_tag: int = 5, magzero: float = 30.0) -> Dict:
    """Sersic components placed uniformly over a large field: mag ~ U[14, 22],
    nser ~ logU[0.5, 8], re ~ logU[1, 60] px, ang ~ U[0, 180], axrat ~ U[0.3, 1];
    Moffat PSF (fwhm 3, con 2.5) with the FFT convolver; all 8 parameters of
    every component in the gradient."""
    r = _rng(seed_tag)
    profs = []
    for _ in range(n_profiles):
        profs.append(("sersic", dict(xcen=r.uniform(0, width), ycen=r.uniform(0, height), mag=r.uniform(14, 22),
                                     nser=float(np.exp(r.uniform(np.log(0.5), np.log(8)))),
                                     re=float(np.exp(r.uniform(0, np.log(60)))), ang=r.uniform(0, 180),
                                     axrat=r.uniform(0.3, 1.0), box=0.0, convolve=True)))
    grad = [(i, k) for i in range(n_profiles) for k in ("xcen", "ycen", "mag", "re", "nser", "ang", "axrat", "box")]
    return dict(name="large_field", width=width, height=height, magzero=magzero,
                psf=moffat_psf(psf_size, 3.0, 2.5), convolver="fft", profiles=profs, grad=grad,
                sigma_range=(1.0, 1.0), seed_tag=seed_tag)


def make_data(w: Dict, model_image: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Data = model + N(0, sigma) with a per-pixel sigma map ~ U[sigma_range]."""
    r = _rng(1000 + w["seed_tag"])
    lo, hi = w["sigma_range"]
    sigma = np.full(model_image.shape, lo) if lo == hi else r.uniform(lo, hi, size=model_image.shape)
    image = model_image + r.normal(0.0, 1.0, size=model_image.shape) * sigma
    return image, sigma


def configure(model, w: Dict):
    """Applies a workload to anything with libprofit's Model methods
    (profit_b200.Model, or the oracle's RefModel / OracleModel)."""
    model.set_magzero(w["magzero"])
    if w.get("psf") is not None:
        model.set_psf(w["psf"])
    model.set_convolver(w.get("convolver", "brute"))
    for name, params in w["profiles"]:
        model.add_profile(name, **params)
    return model


def perturbed(w: Dict, seed: int, scale: float = 0.05) -> Dict:
    """A sampler proposal: params = init + N(0, scale*|init|), redrawn until valid."""
    r = np.random.Generator(np.random.PCG64([SEED, 77, seed]))
    out = dict(w)
    profs = [(name, dict(params)) for name, params in w["profiles"]]
    for idx, k in w["grad"]:
        q = profs[idx][1]
        for _ in range(100):
            v = q[k] + r.normal(0.0, scale * abs(q[k]))
            if {"axrat": 0.05 < v <= 1, "re": v > 0, "nser": v > 0.3, "fwhm": v > 0}.get(k, True):
                q[k] = float(v)
                break
    out["profiles"] = profs
    return out


def catalogue_galaxy_profiles(r: np.random.Generator, side: int) -> List[Tuple[str, Dict]]:
    """1-3 components drawn from the six radial kinds: nser ~ logU[0.5, 10],
    re ~ logU[1, 50] px (capped at the image side), axrat ~ U[0.1, 1],
    ang ~ U[0, 180], box ~ U[-0.3, 0.3].  Non-Sersic kinds map (re, nser) to
    their own parameters: moffat fwhm = re, con = 1 + nser; ferrer rout = 2 re,
    a = 1, b = 1; king rt = 3 re, rc = re, a = 2; brokenexp h1 = re, h2 = re/2,
    rb = 2 re, a = 1; coresersic re, nser, rb = re/4, a = 2, b = 0.5."""
    kinds = ("sersic", "coresersic", "moffat", "ferrer", "king", "brokenexp")
    out = []
    cx, cy = side / 2.0 + r.uniform(-2, 2), side / 2.0 + r.uniform(-2, 2)
    for _ in range(int(r.integers(1, 4))):
        kind = kinds[int(r.integers(0, len(kinds)))]
        nser = float(np.exp(r.uniform(np.log(0.5), np.log(10))))
        re = float(min(np.exp(r.uniform(0, np.log(50))), side / 2.0))
        common = dict(xcen=cx + r.uniform(-1, 1), ycen=cy + r.uniform(-1, 1), mag=float(r.uniform(17, 21)),
                      ang=float(r.uniform(0, 180)), axrat=float(r.uniform(0.1, 1)), box=float(r.uniform(-0.3, 0.3)))
        if kind == "sersic":
            shape = dict(re=re, nser=nser)
        elif kind == "moffat":
            shape = dict(fwhm=re, con=1 + nser)
        elif kind == "ferrer":
            shape = dict(rout=2 * re, a=1.0, b=1.0)
        elif kind == "king":
            shape = dict(rt=3 * re, rc=re, a=2.0)
        elif kind == "brokenexp":
            shape = dict(h1=re, h2=re / 2, rb=2 * re, a=1.0)
        else:
            shape = dict(re=re, nser=nser, rb=re / 4, a=2.0, b=0.5)
        out.append((kind, dict(common, **shape)))
    return out


def catalogue(n: int = 10000, seed_tag: int = 6, side_range=(32, 512), magzero: float = 30.0):
    """Uneven catalogue: n galaxies, square side ~ logU[side_range], per-galaxy
    Gaussian or Moffat PSF of odd side in [15, 65] (FWHM ~ U[2, 4]), profiles as
    catalogue_galaxy_profiles.  Returns a list of dicts (side, psf, profiles);
    data and sigma come from catalogue_data()."""
    r = _rng(seed_tag)
    gals = []
    for _ in range(n):
        side = int(round(np.exp(r.uniform(np.log(side_range[0]), np.log(side_range[1])))))
        psf_side = int(r.integers(7, 33)) * 2 + 1
        fwhm = float(r.uniform(2, 4))
        psf = gaussian_psf(psf_side, fwhm) if r.uniform() < 0.5 else moffat_psf(psf_side, fwhm, 2.5)
        gals.append(dict(side=side, psf=psf, profiles=catalogue_galaxy_profiles(r, side), magzero=magzero))
    return gals
