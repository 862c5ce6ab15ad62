"""The hand-written adjoint of compiled .m models (transposed transforms,
symbolic derivatives of the generated element-wise statements, the implicit
diffusion solve, checkpointed replay), through the C ABI, against central
finite differences of the f64 oracle driving the same IMEX steps.
Tolerance: 1e-4 relative (gradients of the fp32 GPU trajectory vs the f64
trajectory's finite differences, h = 1e-3 relative)."""
import numpy as np
import pytest

from oracle import oracle as O
from turing_sphere_b200 import (GpuModel, ShtConfig, ShtPlan, defaultParams, lmIndex,
                                mModelByKey, nlmCalc)

pytestmark = pytest.mark.gpu

TOL = 1e-4


def spectrum_l2(lmax, seed, amp=0.1, base=0.0):
    """Gaussian coefficients with an l^-2 spectrum (l >= 1), l = 0 set to
    `base` (times sqrt(4 pi)), m = 0 imaginary parts zero."""
    rng = np.random.default_rng(seed)
    q = np.zeros(2 * nlmCalc(lmax, lmax))
    for m in range(lmax + 1):
        for l in range(m, lmax + 1):
            i = lmIndex(lmax, l, m)
            if l == 0:
                q[2 * i] = base * np.sqrt(4 * np.pi)
                continue
            q[2 * i] = amp * rng.standard_normal() / l ** 2
            q[2 * i + 1] = 0.0 if m == 0 else amp * rng.standard_normal() / l ** 2
    return q


def run_oracle(ref, key, params, U0, nsteps):
    return ref.model_step(key, params, np.array(U0, dtype=np.float64), nsteps)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-30)


@pytest.mark.parametrize("precision", ["fp32", "tf32x3"])
def test_allencahn_grid_loss_gradients(device, precision):
    """The Allen-Cahn adjoint workload in small: Allen-Cahn, L = ||u(T) - u_target||^2 on the grid,
    gradients w.r.t. the initial coefficients (two random directions) and
    eps2, with checkpoints every 8 of 20 steps."""
    model = mModelByKey("allencahn")
    lmax, nlat, nphi, nsteps, every = 31, 48, 96, 20, 8
    p = dict(defaultParams(model))
    plist = [p["eps2"], p["dt"]]
    sht = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi), {"precision": precision})
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    U0 = spectrum_l2(lmax, 1, amp=0.5, base=0.1)
    target = ref.synth(spectrum_l2(lmax, 2, amp=0.5, base=-0.1))

    gpu = GpuModel.create(device, sht, model.source, ["eps2", "dt"], ["U"], ["u"], 1)
    gpu.setParams(p)
    gpu.upload("U", U0.astype(np.float32))

    def final_bar(final):
        u = ref.synth(final["U"][0].astype(np.float64))
        gbar = 2.0 * (u - target)
        return {"U": ref.synth_adjoint(gbar)[None, :]}

    init_bar, pbar = gpu.lossGradient(nsteps, every, final_bar)

    def loss(U, prm):
        UT = run_oracle(ref, "allencahn", prm, U[None, :], nsteps)[0]
        return float(((ref.synth(UT) - target) ** 2).sum())

    rng = np.random.default_rng(9)
    for _ in range(2):
        d = spectrum_l2(lmax, int(rng.integers(1 << 30)), amp=1.0)
        h = 1e-3 * np.linalg.norm(U0) / np.linalg.norm(d)
        fd = (loss(U0 + h * d, plist) - loss(U0 - h * d, plist)) / (2 * h)
        ad = float(np.dot(init_bar["U"][0].astype(np.float64), d))
        assert rel(ad, fd) < TOL, (ad, fd)
    h = 1e-3 * plist[0]
    fd = (loss(U0, [plist[0] + h, plist[1]]) - loss(U0, [plist[0] - h, plist[1]])) / (2 * h)
    assert rel(pbar[0, 0], fd) < TOL, (pbar[0, 0], fd)
    # the model ends at the final state, as after step(nsteps)
    UT = run_oracle(ref, "allencahn", plist, U0[None, :], nsteps)[0]
    assert O.rel_l2(gpu.read("U"), UT) < 1e-5


def test_schnakenberg_batched_parameter_gradients(device):
    """The Schnakenberg sweep adjoint in small: two Schnakenberg instances with their own
    parameters, L = sum_k <w_k, (U_T, V_T)_k>; per-instance gradients
    w.r.t. (a, b, D1, D2) and the initial state, checkpoints every 5 of 12."""
    model = mModelByKey("schnakenberg")
    lmax, nlat, nphi, nsteps, every = 31, 48, 96, 12, 5
    base = defaultParams(model)
    names = [q.key for q in model.params]
    sweep = [dict(base, a=base["a"] + 0.02 * k, D1=base["D1"] * (1 + 0.5 * k)) for k in range(2)]
    sht = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi), {"precision": "tf32x3"})
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    gpu = GpuModel.create(device, sht, model.source, names, list(model.state),
                          list(model.species), 2)
    gpu.setParams(sweep)
    rng = np.random.default_rng(4)
    U0 = [np.stack([spectrum_l2(lmax, 10 + 2 * k, 0.05, sweep[k]["a"] + sweep[k]["b"]),
                    spectrum_l2(lmax, 11 + 2 * k, 0.05,
                                sweep[k]["b"] / (sweep[k]["a"] + sweep[k]["b"]) ** 2)])
          for k in range(2)]
    gpu.upload("U", np.stack([u[0] for u in U0]).astype(np.float32))
    gpu.upload("V", np.stack([u[1] for u in U0]).astype(np.float32))
    w = rng.standard_normal((2, 2, 2 * sht.nlm))  # [instance][state]
    init_bar, pbar = gpu.forwardBackward(nsteps, every, {"U": w[:, 0], "V": w[:, 1]})

    def loss(k, U, prm):
        out = run_oracle(ref, "schnakenberg", prm, U, nsteps)
        return float((w[k] * out).sum())

    for k in range(2):
        prm = [sweep[k][n] for n in names]
        for j in range(4):  # a, b, D1, D2
            h = 1e-3 * abs(prm[j])
            up = list(prm); up[j] += h
            dn = list(prm); dn[j] -= h
            fd = (loss(k, U0[k], up) - loss(k, U0[k], dn)) / (2 * h)
            assert rel(pbar[k, j], fd) < TOL, (k, names[j], pbar[k, j], fd)
        d = np.stack([spectrum_l2(lmax, 40 + k, 1.0), spectrum_l2(lmax, 50 + k, 1.0)])
        h = 1e-3 * np.linalg.norm(U0[k]) / np.linalg.norm(d)
        fd = (loss(k, U0[k] + h * d, prm) - loss(k, U0[k] - h * d, prm)) / (2 * h)
        ad = float((init_bar["U"][k] * d[0]).sum() + (init_bar["V"][k] * d[1]).sum())
        assert rel(ad, fd) < TOL, (k, ad, fd)


def test_linear_adjoint_is_exact_transpose(device):
    """For the linear model the step is a linear map G: the adjoint of n
    steps applied to w equals (G^T)^n w, checked through <w, G^n x> =
    <(G^T)^n w, x> on the GPU's own forward map (every = 3 of 7 steps)."""
    src = open(__file__.replace("test_adjoint_gpu.py", "models/linear.m")).read()
    lmax, nlat, nphi, nsteps = 15, 24, 48, 7
    sht = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi), {"precision": "fp32"})
    gpu = GpuModel.create(device, sht, src, ["c", "D", "dt"], ["U"], ["u"], 1)
    gpu.setParams({"c": -0.3, "D": 0.01, "dt": 0.1})
    x = spectrum_l2(lmax, 3, 1.0).astype(np.float32)
    w = spectrum_l2(lmax, 4, 1.0).astype(np.float32)
    gpu.upload("U", x)
    gx = None

    def fb(final):
        nonlocal gx
        gx = final["U"][0].astype(np.float64)
        return {"U": w[None, :]}

    init_bar, _ = gpu.lossGradient(nsteps, 3, fb)
    lhs = float(np.dot(w.astype(np.float64), gx))
    rhs = float(np.dot(init_bar["U"][0].astype(np.float64), x.astype(np.float64)))
    assert rel(lhs, rhs) < 1e-5, (lhs, rhs)
