"""The oracle's f64 adjoint (test infrastructure: the check for the GPU's
hand-written adjoint) pinned on the CPU: its transform adjoints are exact
transposes of its transforms (dot-product identities), and its reverse mode
of whole IMEX runs, for every model, matches central finite differences of
its own f64 forward steps, with and without checkpointing."""
import numpy as np
import pytest

from oracle import oracle as O

LMAX, NLAT, NPHI = 11, 18, 36

PARAMS = {"schnakenberg": [0.1, 0.9, 4e-3, 8e-2, 0.05],
          "brusselator": [3.0, 9.0, 3.33e-2, 1.67e-1, 0.02],
          "allencahn": [1e-2, 0.05],
          "linear": [-0.3, 0.01, 0.1],
          "logistic": [0.7, 0.01, 0.05]}
BASE = {"schnakenberg": (1.0, 0.9), "brusselator": (3.0, 3.0), "allencahn": (0.2,),
        "linear": (0.5,), "logistic": (0.3,)}


def state(ref, key, seed):
    rng = np.random.default_rng(seed)
    st = []
    for b in BASE[key]:
        q = 0.05 * rng.standard_normal(2 * ref.nlm)
        q[0] = b * np.sqrt(4 * np.pi)
        q[1:2 * (LMAX + 1):2] = 0.0
        st.append(q)
    return np.stack(st)


@pytest.fixture(scope="module")
def ref():
    return O.ShtReference(LMAX, LMAX, NLAT, NPHI, threads=1)


def test_transform_adjoints_are_transposes(ref):
    rng = np.random.default_rng(1)
    q = rng.standard_normal(2 * ref.nlm)
    q[1:2 * (LMAX + 1):2] = 0.0
    g = rng.standard_normal(NLAT * NPHI)
    for lhs, rhs in ((np.dot(ref.synth(q), g), np.dot(q, ref.synth_adjoint(g))),
                     (np.dot(ref.analys(g), q), np.dot(g, ref.analys_adjoint(q)))):
        assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


@pytest.mark.parametrize("key", list(PARAMS))
@pytest.mark.parametrize("every", [1, 3, 50])
def test_model_adjoint_matches_central_differences(ref, key, every):
    nsteps = 7
    prm = PARAMS[key]
    x0 = state(ref, key, 2)
    rng = np.random.default_rng(3)
    w = rng.standard_normal(x0.shape)

    def loss(x, p):
        return float((w * ref.model_step(key, p, x, nsteps)).sum())

    ib, pb = ref.model_adjoint(key, prm, x0, nsteps, every, w)
    for j in range(len(prm)):
        h = 1e-6 * abs(prm[j])
        up = list(prm); up[j] += h
        dn = list(prm); dn[j] -= h
        fd = (loss(x0, up) - loss(x0, dn)) / (2 * h)
        assert abs(pb[j] - fd) <= 1e-6 * max(abs(fd), 1e-3), (key, j, pb[j], fd)
    d = state(ref, key, 5)
    d[:, 0] = 0.0
    h = 1e-6 * np.linalg.norm(x0) / np.linalg.norm(d)
    fd = (loss(x0 + h * d, prm) - loss(x0 - h * d, prm)) / (2 * h)
    ad = float((ib * d).sum())
    assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1e-3), (key, ad, fd)
