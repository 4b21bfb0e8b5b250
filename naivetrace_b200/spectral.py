"""Binned spectral helpers on the host (src/spectral.hxx, src/spectral.cxx).

36 bins of 10 nm from 370 to 730 nm.  RGB -> spectrum uses Smits' method with the
reference's basis spectra; spectrum -> RGB uses the reference's 3 x 36 matrix.  The
numbers live in csrc/tt_tables.h; they are parsed from there so that host and device
share one copy.
"""
from __future__ import annotations

import re
from functools import lru_cache
from pathlib import Path

import numpy as np

NBINS = 36
LAMBDA_MIN = 370.0
LAMBDA_MAX = 730.0
WAVELENGTHS = LAMBDA_MIN + 5.0 + 10.0 * np.arange(NBINS)

_TABLES = Path(__file__).resolve().parent / "csrc" / "tt_tables.h"


@lru_cache(maxsize=1)
def tables():
    """(smits[7,36], spectrum_to_rgb[3,36], sun[36]) parsed from csrc/tt_tables.h."""
    text = _TABLES.read_text()

    def grab(name, count):
        m = re.search(r"double " + name + r"[^=]*=\s*\{(.*?)\};", text, re.S)
        nums = [float(x) for x in re.findall(r"-?\d+\.\d+(?:[eE]-?\d+)?", m.group(1))]
        assert len(nums) == count, (name, len(nums))
        return np.array(nums)

    smits = grab("kSmitsBasis", 7 * NBINS).reshape(7, NBINS)
    m = grab("kSpectrumToRgb", 3 * NBINS).reshape(3, NBINS)
    sun = grab("kSunSpectrum", NBINS)
    return smits, m, sun


WHITE, RED, GREEN, BLUE, YELLOW, CYAN, MAGENTA = range(7)


def rgb_to_spectrum(rgb) -> np.ndarray:
    """Smits (2000) as in Color::RGBToSpectrum (spectral.cxx:81-115)."""
    r, g, b = (float(x) for x in rgb)
    s = tables()[0]
    if r <= g and r <= b:
        if g <= b:
            return r * s[WHITE] + (g - r) * s[CYAN] + (b - g) * s[BLUE]
        return r * s[WHITE] + (b - r) * s[CYAN] + (g - b) * s[GREEN]
    if g <= r and g <= b:
        if r <= b:
            return g * s[WHITE] + (r - g) * s[MAGENTA] + (b - r) * s[BLUE]
        return g * s[WHITE] + (b - g) * s[MAGENTA] + (r - b) * s[RED]
    if r <= g:
        return b * s[WHITE] + (r - b) * s[YELLOW] + (g - r) * s[GREEN]
    return b * s[WHITE] + (g - b) * s[YELLOW] + (r - g) * s[RED]


def spectrum_to_rgb(spec) -> np.ndarray:
    return tables()[1] @ np.asarray(spec, dtype=np.float64)


def as_spectrum(x) -> np.ndarray:
    """Scalar -> flat spectrum; length-3 -> Smits RGB spectrum; length-36 -> as is."""
    a = np.asarray(x, dtype=np.float64)
    if a.ndim == 0:
        return np.full(NBINS, float(a))
    if a.shape == (3,):
        return rgb_to_spectrum(a)
    if a.shape == (NBINS,):
        return a
    raise ValueError(f"cannot interpret {a.shape} as a spectrum")


def band_spectrum(inside: float, outside: float, lo_bin: int, hi_bin: int) -> np.ndarray:
    s = np.full(NBINS, outside)
    s[lo_bin:hi_bin + 1] = inside
    return s
