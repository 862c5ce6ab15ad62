"""Grid and spectral layout (src/sht/layout.ts of the reference).

Spectral coefficients Q_lm: complex, m >= 0 only, interleaved [re, im],
m-major order lm(l, m) = m(lmax+1) - m(m-1)/2 + (l-m).  Spatial fields:
real, spat[ilat*nphi + iphi], ilat north to south.  Orthonormal harmonics
with the Condon-Shortley phase; m = 0 coefficients have zero imaginary part.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _lib


@dataclass(frozen=True)
class ShtConfig:
    lmax: int
    mmax: int
    nlat: int
    nphi: int


def nlmCalc(lmax: int, mmax: int) -> int:
    """layout.ts:24-27"""
    return int(_lib.lib().ts_nlm_calc(lmax, mmax))


def lmIndex(lmax: int, l: int, m: int) -> int:
    """layout.ts:30-32"""
    return int(_lib.lib().ts_lm_index(lmax, l, m))


def validateConfig(cfg: ShtConfig) -> None:
    """layout.ts:34-44: raises ValueError with the reference's message."""
    for k in ("lmax", "mmax", "nlat", "nphi"):
        if int(getattr(cfg, k)) != getattr(cfg, k):
            raise ValueError(f"{k} must be an integer (got {getattr(cfg, k)})")
    buf = C.create_string_buffer(256)
    rc = _lib.lib().ts_validate_config(cfg.lmax, cfg.mmax, cfg.nlat, cfg.nphi, buf, 256)
    if rc != _lib.TS_OK:
        raise ValueError(buf.value.decode())


def isPowerOfTwo(n: int) -> bool:
    return n > 0 and (n & (n - 1)) == 0


def gridForLmax(lmax: int, pdeg: int) -> tuple[int, int]:
    """layout.ts:53-59: (nlat, nphi) dealiased for a degree-pdeg reaction."""
    a, b = C.c_int(), C.c_int()
    _lib.lib().ts_grid_for_lmax(lmax, pdeg, C.byref(a), C.byref(b))
    return a.value, b.value


def gaussGrid(lmax: int) -> tuple[int, int]:
    """The 3(lmax+1)/2 x 2*nlat Gauss grid (nlat rounded up to even), the
    grid family of the large configurations (nphi = 3*2^k when lmax+1 is a
    power of two, which the mixed-radix FFT covers)."""
    nlat = (3 * (lmax + 1) + 1) // 2
    nlat += nlat & 1
    return nlat, 2 * nlat
