"""Compiled .m models on the GPU, through the C ABI: the reference's analytic
checks (test/analyticChecks.ts), its model checks (test/modelChecks.ts), and
parity of whole IMEX runs with the f64 oracle driving the same step."""
import math
import os

import numpy as np
import pytest

from oracle import oracle as O
from turing_sphere_b200 import (GpuModel, ModelGroup, ModelSession, ShtConfig, ShtPlan,
                                defaultParams,
                                gridForLmax, lmIndex, mModelByKey, mModels, nlmCalc, seededNoise)
from turing_sphere_b200.registry import MModel, ParamSpec

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
LINEAR = open(os.path.join(HERE, "models", "linear.m")).read()
LOGISTIC = open(os.path.join(HERE, "models", "logistic.m")).read()


def make(device, source, params, lmax, pdeg, state=("U",), view=("u",), batch=1, grid=None):
    nlat, nphi = grid if grid else gridForLmax(lmax, pdeg)
    sht = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi))
    gpu = GpuModel.create(device, sht, source, params, list(state), list(view), batch)
    return sht, gpu


def test_A_linear_reaction_exact_growth(device):
    """analyticChecks.ts:74-122."""
    lmax, c, D, dt, n = 15, -0.3, 0.01, 0.1, 20
    sht, gpu = make(device, LINEAR, ["c", "D", "dt"], lmax, 1)
    gpu.setParams({"c": c, "D": D, "dt": dt})
    nlm = nlmCalc(lmax, lmax)
    l, m = 5, 2
    idx = lmIndex(lmax, l, m)
    U0 = np.zeros(2 * nlm, dtype=np.float32)
    U0[2 * idx], U0[2 * idx + 1] = 0.8, -0.35
    gpu.upload("U", U0)
    gpu.step(n)
    U = gpu.read("U")
    g = ((1 + dt * c) / (1 + dt * D * l * (l + 1))) ** n
    assert abs(U[2 * idx] - 0.8 * g) < 2e-6 and abs(U[2 * idx + 1] + 0.35 * g) < 2e-6
    other = np.delete(U.reshape(-1, 2), idx, axis=0)
    assert np.abs(other).max() < 2e-6


def test_B_logistic_uniform_field(device):
    """analyticChecks.ts:125-181."""
    lmax, r, D, dt, n, u0 = 15, 0.7, 0.01, 0.05, 25, 0.3
    sht, gpu = make(device, LOGISTIC, ["r", "D", "dt"], lmax, 3)
    gpu.setParams({"r": r, "D": D, "dt": dt})
    npts = sht.cfg.nlat * sht.cfg.nphi
    gpu.init(np.full(npts, u0, dtype=np.float32))
    Us = gpu.read("U")
    gpu.step(n)
    Ue = gpu.read("U")
    got = u0 * (Ue[0] / Us[0])
    want = u0
    for _ in range(n):
        want += dt * r * want * (1 - want)
    assert abs(got - want) < 5e-6, (got, want)
    u = gpu.read("u")
    assert u.max() - u.min() < 1e-6


def test_C_schnakenberg_linearised_recurrence(device):
    """analyticChecks.ts:184-256."""
    model = mModelByKey("schnakenberg")
    p = defaultParams(model)
    lmax = 31
    sht, gpu = make(device, model.source, [q.key for q in model.params], lmax, model.pdeg,
                    model.state, model.species)
    gpu.setParams(p)
    npts = sht.cfg.nlat * sht.cfg.nphi
    gpu.init(np.zeros(npts, dtype=np.float32))
    l, m, eps = 24, 7, 1e-6
    idx = lmIndex(lmax, l, m)
    U0, V0 = gpu.read("U"), gpu.read("V")
    Up = U0.copy()
    Up[2 * idx] += eps
    gpu.upload("U", Up)
    gpu.upload("V", V0)
    n = 40
    gpu.step(n)
    U, V = gpu.read("U"), gpu.read("V")
    us = p["a"] + p["b"]
    vs = p["b"] / (us * us)
    J = [[-1 + 2 * us * vs, us * us], [-2 * us * vs, -us * us]]
    lam = l * (l + 1)
    du, dv = 1 / (1 + p["dt"] * p["D1"] * lam), 1 / (1 + p["dt"] * p["D2"] * lam)
    cu, cv = eps, 0.0
    for _ in range(n):
        cu, cv = ((cu + p["dt"] * (J[0][0] * cu + J[0][1] * cv)) * du,
                  (cv + p["dt"] * (J[1][0] * cu + J[1][1] * cv)) * dv)
    gu, gv = U[2 * idx] - U0[2 * idx], V[2 * idx] - V0[2 * idx]
    assert abs(gu - cu) / abs(cu) < 5e-3 and abs(gv - cv) / abs(cv) < 5e-3
    assert abs(cu) > eps and abs(gu) > eps


@pytest.mark.parametrize("model", mModels, ids=lambda m: m.key)
def test_models_run_finite_and_patterned(device, model):
    """modelChecks.ts:56-77: lmax 31, seed 1, 40 steps."""
    s = ModelSession.create(device, model, defaultParams(model), 31)
    kernels, launches = s.gpu.counts("step")
    assert kernels == {"schnakenberg": 5, "brusselator": 5, "allencahn": 2}[model.key]
    assert launches == 3
    s.seed(1)
    s.step(40)
    for f in model.species:
        v = s.read(f)
        assert np.isfinite(v).all() and v.max() - v.min() > 1e-6
    s.destroy()


def test_view_reads_synth_of_previous_state(device):
    """`u = synth(U)` runs before the update, so after a step the displayed
    field is the synthesis of the state the step started from."""
    model = mModelByKey("allencahn")
    s = ModelSession.create(device, model, defaultParams(model), 31)
    s.seed(3)
    s.step(5)
    U_before = s.read("U")
    s.step(1)
    u = s.read("u")
    want = s.sht.synth(U_before)
    assert np.abs(u - want).max() < 1e-6
    s.destroy()


def test_oversample_measure_and_setoversample(device):
    """modelChecks.ts:82-169."""
    model = mModelByKey("allencahn")
    s = ModelSession.create(device, model, defaultParams(model), 31, oversample=2)
    s.seed(1)
    s.step(40)
    fine = s.readSpecies(0)
    d = s.viewSht.cfg
    assert d.nlat == 2 * s.cfg.nlat and d.nphi == 2 * s.cfg.nphi and fine.size == d.nlat * d.nphi
    q = s.read("U")
    assert np.abs(fine - s.viewSht.synth(q)).max() <= 1e-6
    t0, n0 = s.t, s.steps
    s.measure(8)
    after = s.read("U")
    assert np.array_equal(q, after) and s.t == t0 and s.steps == n0
    s.setOversample(1)
    assert np.array_equal(s.read("U"), after) and s.viewSht is s.sht
    s.step(1)
    assert s.readSpecies(0).size == s.cfg.nlat * s.cfg.nphi
    s.destroy()


def spectral_seed(lmax, p, seed, amp=1e-2):
    """Spectral seeding of the single-instance run: the homogeneous state u* = a+b, v* = b/(a+b)^2 in the
    l = 0 coefficient (times sqrt(4 pi)) plus N(0, amp^2) on every
    coefficient with 1 <= l <= lmax (m = 0 imaginary parts zero)."""
    rng = np.random.default_rng(seed)
    nlm = nlmCalc(lmax, lmax)
    us = p["a"] + p["b"]
    vs = p["b"] / (us * us)
    out = []
    for base in (us, vs):
        q = (amp * rng.standard_normal(2 * nlm)).astype(np.float32)
        # m = 0 comes first in m-major order: lm(l, 0) = l, so (l, m) = (0, 0) is lm 0
        q[0] = base * math.sqrt(4 * math.pi)
        q[1:2 * (lmax + 1):2] = 0.0
        out.append(q)
    return out


@pytest.mark.parametrize("nsteps", [20, 1000])
def test_schnakenberg_run_matches_f64_oracle(device, nsteps):
    """A single Schnakenberg instance (lmax 63, 96 x 192 Gauss grid): the fp32 GPU run against the
    f64 oracle driving the same IMEX step; <= 1e-4 relative L2 per field."""
    model = mModelByKey("schnakenberg")
    p = defaultParams(model)
    lmax, nlat, nphi = 63, 96, 192
    s = ModelSession.create(device, model, p, lmax, grid=(nlat, nphi))
    U0, V0 = spectral_seed(lmax, p, 1)
    s.gpu.upload("U", U0)
    s.gpu.upload("V", V0)
    s.step(nsteps)
    U, V = s.read("U"), s.read("V")
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    out = ref.model_step("schnakenberg", [p["a"], p["b"], p["D1"], p["D2"], p["dt"]],
                         np.stack([U0, V0]).astype(np.float64), nsteps)
    eU, eV = O.rel_l2(U, out[0]), O.rel_l2(V, out[1])
    assert eU < 1e-4 and eV < 1e-4, (eU, eV)
    s.destroy()


@pytest.mark.parametrize("lmax,grid,batch,nsteps,check",
                         [(63, (96, 192), 4, 40, (0, 1, 2, 3)),
                          (63, (96, 192), 12, 40, (0, 5, 11)),
                          (255, (384, 768), 12, 2, (0, 11))])
def test_tc_batched_imex_matches_f64_oracle(device, lmax, grid, batch, nsteps, check):
    """Batched Schnakenberg IMEX on the tensor-core plan (a sweep over b,
    spectral seed 1 + k for instance k) against the f64 oracle stepping each
    instance alone.  Up to 16 instance-fields the IMEX update runs in the
    analysis kernel's epilogue, above that as its own element-wise kernel:
    batches 4 and 12 (8 and 24 fields) cover both.  <= 1e-4 relative L2 per
    field, the bound of the FP32 single-instance run."""
    model = mModelByKey("schnakenberg")
    base = defaultParams(model)
    sweep = [dict(base, b=base["b"] + 0.01 * k) for k in range(batch)]
    s = ModelSession.create(device, model, sweep, lmax, batch=batch, grid=grid,
                            precision="tf32x3")
    seeds = [spectral_seed(lmax, sweep[k], 1 + k) for k in range(batch)]
    s.gpu.upload("U", np.stack([q[0] for q in seeds]))
    s.gpu.upload("V", np.stack([q[1] for q in seeds]))
    s.step(nsteps)
    U, V = s.read("U"), s.read("V")
    s.destroy()
    ref = O.ShtReference(lmax, lmax, grid[0], grid[1])
    for k in check:
        p = sweep[k]
        out = ref.model_step("schnakenberg", [p["a"], p["b"], p["D1"], p["D2"], p["dt"]],
                             np.stack(seeds[k]).astype(np.float64), nsteps)
        eU, eV = O.rel_l2(U[k], out[0]), O.rel_l2(V[k], out[1])
        assert eU < 1e-4 and eV < 1e-4, (k, eU, eV)


def test_batched_sweep_equals_single_instances(device):
    """Per-instance parameters (a Brusselator (A, B) sweep): each instance of
    one batched model equals the same instance run alone."""
    model = mModelByKey("brusselator")
    base = defaultParams(model)
    sweep = [dict(base, A=2.8 + 0.1 * k, B=7.0 + 0.5 * k) for k in range(4)]
    lmax = 31
    batched = ModelSession.create(device, model, sweep, lmax, batch=4)
    batched.seed(10)
    batched.step(30)
    Ub = batched.read("U")
    for k in (0, 3):
        single = ModelSession.create(device, model, sweep[k], lmax)
        single.seed(10 + k)
        single.step(30)
        assert O.rel_l2(Ub[k], single.read("U")) < 1e-6
        single.destroy()
    batched.destroy()


def test_snapshot_restore_is_exact(device):
    model = mModelByKey("schnakenberg")
    s = ModelSession.create(device, model, defaultParams(model), 31)
    s.seed(2)
    s.step(3)
    U = s.read("U")
    s.gpu.snapshotState()
    s.gpu.step(7)
    assert not np.array_equal(s.read("U"), U)
    s.gpu.restoreState()
    assert np.array_equal(s.read("U"), U)
    s.destroy()


@pytest.mark.parametrize("precision", ["fp32", "tf32x3"])
def test_graph_steps_equal_eager_steps(device, precision):
    """Steps replayed from captured CUDA graphs (pairs of steps at both state
    parities and a single step for an odd count) give bit-identical states
    to eagerly launched steps."""
    model = mModelByKey("brusselator")
    p = defaultParams(model)
    lmax = 31
    nlat, nphi = gridForLmax(lmax, model.pdeg)
    sht = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi), {"precision": precision})
    out = []
    for graphs in (True, False):  # the context's own (capturable) stream
        gpu = GpuModel.create(device, sht, model.source, [q.key for q in model.params],
                              list(model.state), list(model.species), 3)
        gpu.setGraphs(graphs)
        gpu.setParams([dict(p, A=p["A"] + 0.1 * k) for k in range(3)])
        gpu.init(np.concatenate([seededNoise(nlat * nphi, model.seedAmp, 7 + k)
                                 for k in range(3)]))
        for n in (1, 4, 3, 2, 5):  # eager warm-up, then graphs at both parities
            gpu.step(n)
        out.append((gpu.read("U"), gpu.read("V"), gpu.read("u")))
        gpu.destroy()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_ragged_group_equals_separate_models(device):
    """A ragged batch (Brusselator instances at lmax 15, 31 and 63 on their
    own plans) stepped as one group (concurrent branches in one graph per
    step) ends bit-identical to the same models stepped one by one."""
    model = mModelByKey("brusselator")
    base = defaultParams(model)
    names = [q.key for q in model.params]
    specs = [(15, 2), (31, 3), (63, 1)]

    def build():
        out = []
        for lmax, ni in specs:
            nlat, nphi = gridForLmax(lmax, model.pdeg)
            sht = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi),
                                 {"precision": "tf32x3"})
            gpu = GpuModel.create(device, sht, model.source, names, list(model.state),
                                  list(model.species), ni)
            gpu.setParams([dict(base, A=base["A"] + 0.05 * k) for k in range(ni)])
            gpu.init(np.concatenate([seededNoise(nlat * nphi, model.seedAmp, 3 + k)
                                     for k in range(ni)]))
            out.append((sht, gpu))
        return out

    grouped, single = build(), build()
    group = ModelGroup([g for _, g in grouped])
    for n in (1, 2, 3, 2):  # eager warm-up, then graphs at both parities
        group.step(n)
    for _, g in single:
        g.step(8)
    for (_, a), (_, b) in zip(grouped, single):
        assert np.array_equal(a.read("U"), b.read("U"))
        assert np.array_equal(a.read("V"), b.read("V"))
    group.destroy()
    for _, g in grouped + single:
        g.destroy()


def test_upload_and_read_errors(device):
    model = mModelByKey("allencahn")
    s = ModelSession.create(device, model, defaultParams(model), 15)
    with pytest.raises(ValueError, match="expected"):
        s.gpu.upload("U", np.zeros(3, dtype=np.float32))
    with pytest.raises(ValueError, match="no buffer named"):
        s.gpu.upload("nope", np.zeros(3, dtype=np.float32))
    with pytest.raises(KeyError):
        s.read("nope")
    s.destroy()
