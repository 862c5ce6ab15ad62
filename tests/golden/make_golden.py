"""Generate the golden fixtures in this folder.

Independent sources only:
  * spherical harmonics from scipy.special.sph_harm_y (orthonormal, with the
    Condon-Shortley phase: the convention of layout.ts:10-15);
  * Gauss-Legendre nodes/weights from numpy.polynomial.legendre.leggauss;
  * seeding, grid rule and reaction arithmetic from the reference's own
    bench/shtns/spec.h, compiled from its sources into oracle/_ref by
    oracle/Makefile (run `make -C oracle ref` first, in a tree that has the
    reference checked out).

Run from the repository root:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import scipy.special as sp

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import oracle as O  # noqa: E402


def lm_index(lmax, l, m):
    return m * (lmax + 1) - m * (m - 1) // 2 + (l - m)


def field_from_modes(lmax, modes, theta, nphi):
    """f(theta_i, phi_j) = sum_{m>=0} Q_lm Y_lm + c.c.(m>0), by scipy."""
    phi = 2 * np.pi * np.arange(nphi) / nphi
    TH, PH = np.meshgrid(theta, phi, indexing="ij")
    f = np.zeros_like(TH)
    for (l, m, re, im) in modes:
        y = sp.sph_harm_y(l, m, TH, PH)
        q = re + 1j * im
        f += (q * y).real if m == 0 else 2.0 * (q * y).real
    return f


def main():
    out = {}
    rng = np.random.default_rng(20261203)

    # 1. sph_harm fields on Gauss grids, sparse random spectra
    cases = []
    for lmax, nlat, nphi, nmodes in ((15, 16, 32, 6), (31, 48, 96, 10), (40, 64, 96, 8)):
        x, _ = np.polynomial.legendre.leggauss(nlat)
        theta = np.arccos(x[::-1])  # north -> south
        modes = []
        for _ in range(nmodes):
            l = int(rng.integers(0, lmax + 1))
            m = int(rng.integers(0, l + 1))
            re = float(rng.normal())
            im = 0.0 if m == 0 else float(rng.normal())
            modes.append((l, m, re, im))
        # merge duplicates so the spectrum is well defined
        merged = {}
        for (l, m, re, im) in modes:
            a, b = merged.get((l, m), (0.0, 0.0))
            merged[(l, m)] = (a + re, b + im)
        modes = [(l, m, re, im) for (l, m), (re, im) in sorted(merged.items())]
        f = field_from_modes(lmax, modes, theta, nphi)
        cases.append({"lmax": lmax, "mmax": lmax, "nlat": nlat, "nphi": nphi,
                      "modes": modes, "field": f.ravel().tolist()})
    out["sph_harm_fields"] = cases

    # 2. Gauss-Legendre nodes (decreasing) and weights
    gl = []
    for n in (16, 48, 96, 193):
        x, w = np.polynomial.legendre.leggauss(n)
        gl.append({"n": n, "x": x[::-1].tolist(), "w": w[::-1].tolist()})
    out["gauss"] = gl

    # 3. the reference's spec.h, compiled from its sources
    R = O.SpecRef()
    out["spec_grid"] = [{"lmax": l, "pdeg": p, "grid": list(R.grid_for_lmax(l, p))}
                        for l in (15, 31, 63, 127, 255) for p in (1, 3)]
    out["spec_noise"] = [{"seed": s, "amp": 1e-2, "values": R.seeded_noise(512, 1e-2, s).tolist()}
                         for s in (1, 7)]
    out["spec_spectrum"] = [{"lmax": 15, "seed": s, "values": R.seeded_spectrum(15, 15, s).tolist()}
                            for s in (1, 2)]
    u = np.linspace(-1.5, 3.5, 41).astype(np.float32)
    v = np.linspace(0.1, 1.2, 41).astype(np.float32)
    react = []
    for model in (0, 1, 2):
        r1, r2 = R.react(model, u, v if model < 2 else None)
        react.append({"model": model, "u": u.tolist(), "v": v.tolist(), "r1": r1.tolist(),
                      "r2": None if r2 is None else r2.tolist(),
                      "params": R.default_params(model)})
    out["spec_react_f32"] = react

    path = os.path.join(HERE, "golden.json")
    with open(path, "w") as fh:
        json.dump(out, fh)
    print(f"wrote {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
