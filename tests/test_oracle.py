"""The oracle (f64 C restatement) pinned against independent sources and the
reference's own compiled spec.h.  CPU only."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def spectrum_from_modes(lmax, modes):
    q = np.zeros(2 * O.nlm_calc(lmax, lmax))
    for l, m, re, im in modes:
        i = O.lm_index(lmax, l, m)
        q[2 * i] = re
        q[2 * i + 1] = im
    return q


@pytest.mark.parametrize("case", range(len(GOLDEN["sph_harm_fields"])))
def test_synth_matches_scipy_sph_harm(case):
    c = GOLDEN["sph_harm_fields"][case]
    ref = O.ShtReference(c["lmax"], c["mmax"], c["nlat"], c["nphi"])
    q = spectrum_from_modes(c["lmax"], c["modes"])
    f = ref.synth(q)
    want = np.array(c["field"])
    assert np.abs(f - want).max() < 1e-12 * max(1.0, np.abs(want).max())
    # and the analysis recovers the spectrum exactly (Gauss quadrature)
    assert O.rel_l2(ref.analys(want), q) < 1e-13


@pytest.mark.parametrize("case", range(len(GOLDEN["gauss"])))
def test_gauss_matches_numpy_leggauss(case):
    g = GOLDEN["gauss"][case]
    x, w = O.gauss(g["n"])
    assert np.abs(x - np.array(g["x"])).max() < 1e-15
    assert np.abs(w - np.array(g["w"])).max() < 1e-14


def test_grid_rule_matches_reference_spec_h():
    for e in GOLDEN["spec_grid"]:
        assert list(O.grid_for_lmax(e["lmax"], e["pdeg"])) == e["grid"]


def test_seeding_matches_reference_spec_h():
    for e in GOLDEN["spec_noise"]:
        got = O.seeded_noise(len(e["values"]), e["amp"], e["seed"])
        assert np.array_equal(got, np.array(e["values"], dtype=np.float32))
    for e in GOLDEN["spec_spectrum"]:
        got = O.seeded_spectrum(e["lmax"], e["lmax"], e["seed"])
        assert np.array_equal(got, np.array(e["values"], dtype=np.float32))


@pytest.mark.skipif(not O.SpecRef.available(), reason="oracle/_ref not built")
def test_seeding_matches_reference_live():
    R = O.SpecRef()
    for seed in (1, 3, 99):
        assert np.array_equal(R.seeded_noise(4096, 1e-2, seed), O.seeded_noise(4096, 1e-2, seed))
        assert np.array_equal(R.seeded_spectrum(31, 31, seed), O.seeded_spectrum(31, 31, seed))


def test_random_spectrum_is_real_at_m0():
    q = O.random_spectrum(31, 31, 42)
    for l in range(32):
        assert q[2 * O.lm_index(31, l, 0) + 1] == 0.0
    assert np.all(np.abs(q) <= 1.0)


def test_validate_rules():
    assert O.validate(31, 31, 32, 64) == 0
    assert O.validate(0, 0, 4, 4) == 1
    assert O.validate(31, 32, 48, 96) == 2
    assert O.validate(31, 31, 31, 96) == 3
    assert O.validate(31, 31, 48, 62) == 4


@pytest.mark.parametrize("lmax", [15, 31, 63])
def test_round_trip_identity(lmax):
    nlat, nphi = O.grid_for_lmax(lmax, 3)
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    q = O.seeded_spectrum(lmax, lmax, 1).astype(np.float64)
    assert O.rel_l2(ref.analys(ref.synth(q)), q) < 1e-13


def test_oracle_analytic_linear_growth():
    """Analytic test A (test/analyticChecks.ts:74-122) on the oracle."""
    lmax = 15
    nlat, nphi = O.grid_for_lmax(lmax, 1)
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    c, D, dt, n = -0.3, 0.01, 0.1, 20
    l, m = 5, 2
    idx = O.lm_index(lmax, l, m)
    U = np.zeros(2 * ref.nlm)
    U[2 * idx], U[2 * idx + 1] = 0.8, -0.35
    out = ref.model_step("linear", [c, D, dt], U, n)[0]
    g = ((1 + dt * c) / (1 + dt * D * l * (l + 1))) ** n
    assert abs(out[2 * idx] - 0.8 * g) < 1e-13
    assert abs(out[2 * idx + 1] + 0.35 * g) < 1e-13
    other = np.delete(out.reshape(-1, 2), idx, axis=0)
    assert np.abs(other).max() < 1e-13


def test_oracle_reaction_matches_spec_h():
    for e in GOLDEN["spec_react_f32"]:
        model = e["model"]
        u = np.array(e["u"], dtype=np.float64)
        v = np.array(e["v"], dtype=np.float64)
        p = e["params"]
        if model == 0:
            uuv = u * u * v
            r1, r2 = p["a"] - u + uuv, p["b"] - uuv
        elif model == 1:
            uuv = u * u * v
            r1, r2 = p["a"] - (p["b"] + 1) * u + uuv, p["b"] * u - uuv
        else:
            r1, r2 = u - u * u * u, None
        assert np.allclose(r1, np.array(e["r1"]), rtol=1e-6, atol=1e-6)
        if r2 is not None:
            assert np.allclose(r2, np.array(e["r2"]), rtol=1e-6, atol=1e-6)


def test_oracle_synth_adjoint_is_the_transpose():
    """<synth q, g> = <q, synth_adjoint g> in f64 (the helper the adjoint
    tests form their grid-loss cotangents with)."""
    lmax, nlat, nphi = 15, 24, 48
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    rng = np.random.default_rng(3)
    q = rng.standard_normal(2 * ref.nlm)
    for l in range(lmax + 1):
        q[2 * O.lm_index(lmax, l, 0) + 1] = 0.0
    g = rng.standard_normal(nlat * nphi)
    lhs = float(np.dot(ref.synth(q), g))
    rhs = float(np.dot(q, ref.synth_adjoint(g)))
    assert abs(lhs - rhs) < 1e-10 * max(1.0, abs(lhs))
