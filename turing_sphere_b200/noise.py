"""Seeded perturbations (src/mgpu/noise.ts): mulberry32 + Box-Muller, drawn by
the C library so the integer state matches the reference bit for bit."""
from __future__ import annotations

import numpy as np

from . import _lib


def seededNoise(npts: int, amp: float, seed: int) -> np.ndarray:
    out = np.empty(npts, dtype=np.float32)
    _lib.lib().ts_seeded_noise(npts, amp, seed & 0xFFFFFFFF, _lib.fptr(out))
    return out


def seededSpectrum(lmax: int, mmax: int, seed: int) -> np.ndarray:
    nlm = (mmax + 1) * (lmax + 1) - mmax * (mmax + 1) // 2
    out = np.empty(2 * nlm, dtype=np.float32)
    _lib.lib().ts_seeded_spectrum(lmax, mmax, seed & 0xFFFFFFFF, _lib.fptr(out))
    return out
