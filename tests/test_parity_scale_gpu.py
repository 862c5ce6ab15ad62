"""The tensor-core (split-TF32) model step against the f64 oracle at the sizes
of the benchmark's workloads, through the C ABI.

Every case starts the GPU run and the oracle from the same state (read back
after the GPU's `init`, or uploaded) and advances both the same number of
IMEX steps (the oracle restates the .m op order in f64: synth every species,
the reaction on the grid, analys, the implicit diffusion solve; oracle
model 0 = schnakenberg.m:23-29, model 1 = brusselator.m:22-28).  Bars: 1e-4
relative L2 per field after the run (the single-instance bar), 1e-5 per
transform; short runs also check the state's increment over the run, which
is what the steps computed, against the oracle's increment.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.test_model_gpu import spectral_seed
from turing_sphere_b200 import (GpuModel, ModelGroup, ModelSession, ShtConfig, ShtPlan,
                                defaultParams, mModelByKey, seededNoise)
from turing_sphere_b200.registry import brusselatorSweep

pytestmark = pytest.mark.gpu

FIELD_BAR = 1e-4
TRANSFORM_BAR = 1e-5


def _prm(model_key, p):
    if model_key == "schnakenberg":
        return [p["a"], p["b"], p["D1"], p["D2"], p["dt"]]
    return [p["A"], p["B"], p["D1"], p["D2"], p["dt"]]


def test_tc_schnakenberg_1000_steps_matches_f64_oracle(device, parity):
    """Four Schnakenberg instances (a sweep over b, spectral seed 1 + k) at
    lmax 63 on 96 x 192, tensor-core plan, 1000 steps as captured step
    graphs: instances 0 and 3 against the oracle stepping each alone."""
    model = mModelByKey("schnakenberg")
    base = defaultParams(model)
    lmax, grid, batch, nsteps = 63, (96, 192), 4, 1000
    sweep = [dict(base, b=base["b"] + 0.01 * k) for k in range(batch)]
    s = ModelSession.create(device, model, sweep, lmax, batch=batch, grid=grid,
                            precision="tf32x3")
    seeds = [spectral_seed(lmax, sweep[k], 1 + k) for k in range(batch)]
    s.gpu.upload("U", np.stack([q[0] for q in seeds]))
    s.gpu.upload("V", np.stack([q[1] for q in seeds]))
    s.step(nsteps)
    U, V = s.read("U"), s.read("V")
    s.destroy()
    ref = O.ShtReference(lmax, lmax, *grid)
    for k in (0, 3):
        out = ref.model_step("schnakenberg", _prm("schnakenberg", sweep[k]),
                             np.stack(seeds[k]).astype(np.float64), nsteps)
        parity(f"schnakenberg lmax63 tf32x3 1000 steps inst{k} U", O.rel_l2(U[k], out[0]),
               FIELD_BAR)
        parity(f"schnakenberg lmax63 tf32x3 1000 steps inst{k} V", O.rel_l2(V[k], out[1]),
               FIELD_BAR)


def test_brusselator_sweep_lmax127_matches_f64_oracle(device, parity):
    """The Brusselator sweep workload: 256 instances with (A, B) drawn over
    the Turing-unstable band, lmax 127 on 192 x 384, tensor-core plan, seeded
    grid noise (seed 1 + k) through `init`, then 200 steps.  The state `init`
    produced is checked against the oracle's analysis of the same grids, and
    three instances' runs against the oracle's."""
    model = mModelByKey("brusselator")
    lmax, nlat, nphi, ni, nsteps = 127, 192, 384, 256, 200
    sweep = brusselatorSweep(ni, seed=3)
    sht = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi), {"precision": "tf32x3"})
    gpu = GpuModel.create(device, sht, model.source, [q.key for q in model.params],
                          model.state, model.species, ni)
    gpu.setParams(sweep)
    npts = nlat * nphi
    noise = [seededNoise(npts, model.seedAmp, 1 + k) for k in range(ni)]
    gpu.init(np.concatenate(noise))
    U0, V0 = gpu.read("U"), gpu.read("V")
    gpu.step(nsteps)
    U, V = gpu.read("U"), gpu.read("V")
    gpu.destroy()
    sht.destroy()
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    for k in (0, 255):
        A, B = sweep[k]["A"], sweep[k]["B"]
        u_init = ref.analys(A + noise[k].astype(np.float64))
        v_init = ref.analys(np.full(npts, B / A))
        parity(f"brusselator lmax127 init inst{k} U", O.rel_l2(U0[k], u_init), TRANSFORM_BAR)
        parity(f"brusselator lmax127 init inst{k} V", O.rel_l2(V0[k], v_init), TRANSFORM_BAR)
    for k in (0, 101, 255):
        out = ref.model_step("brusselator", _prm("brusselator", sweep[k]),
                             np.stack([U0[k], V0[k]]).astype(np.float64), nsteps)
        parity(f"brusselator sweep lmax127 200 steps inst{k} U", O.rel_l2(U[k], out[0]),
               FIELD_BAR)
        parity(f"brusselator sweep lmax127 200 steps inst{k} V", O.rel_l2(V[k], out[1]),
               FIELD_BAR)


def test_ragged_group_matches_f64_oracle(device, parity):
    """The ragged workload: 64 Brusselator instances at each of lmax
    63/127/255 (96 x 192, 192 x 384, 384 x 768), one model per lmax on its
    own tensor-core plan, advanced as one model group (captured group graphs)
    for 100 steps; one instance per lmax against the oracle."""
    model = mModelByKey("brusselator")
    p = defaultParams(model)
    names = [q.key for q in model.params]
    parts, starts = [], []
    for lmax, nlat in ((63, 96), (127, 192), (255, 384)):
        sht = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, 2 * nlat),
                             {"precision": "tf32x3"})
        gpu = GpuModel.create(device, sht, model.source, names, list(model.state),
                              list(model.species), 64)
        gpu.setParams(p)
        gpu.init(np.concatenate([seededNoise(nlat * 2 * nlat, model.seedAmp, 1 + k)
                                 for k in range(64)]))
        starts.append((gpu.read("U"), gpu.read("V")))
        parts.append((lmax, nlat, sht, gpu))
    group = ModelGroup([g for *_, g in parts])
    nsteps = 100
    for n in (1, 1, 2, 96):  # eager warm-up steps, then graphs at both parities
        group.step(n)
    group.destroy()
    for (lmax, nlat, sht, gpu), (U0, V0), k in zip(parts, starts, (0, 31, 63)):
        U, V = gpu.read("U"), gpu.read("V")
        ref = O.ShtReference(lmax, lmax, nlat, 2 * nlat)
        out = ref.model_step("brusselator", _prm("brusselator", p),
                             np.stack([U0[k], V0[k]]).astype(np.float64), nsteps)
        parity(f"ragged group lmax{lmax} 100 steps inst{k} U", O.rel_l2(U[k], out[0]), FIELD_BAR)
        parity(f"ragged group lmax{lmax} 100 steps inst{k} V", O.rel_l2(V[k], out[1]), FIELD_BAR)
        gpu.destroy()
        sht.destroy()


def test_schnakenberg_lmax511_batch64_forward_matches_f64_oracle(device, parity):
    """The lmax-511 inverse-problem workload's forward pass: 64 Schnakenberg
    instances (a sweep over D1, spectral seed 1 + k) on 768 x 1536, tensor-core
    plan, 4 steps; instances 0 and 63 against the oracle.  Besides the state,
    the increment U(4) - U(0) the steps produced is held to the field bar."""
    model = mModelByKey("schnakenberg")
    base = defaultParams(model)
    lmax, grid, ni, nsteps = 511, (768, 1536), 64, 4
    sweep = [dict(base, D1=base["D1"] * (1 + 0.5 * k / ni)) for k in range(ni)]
    s = ModelSession.create(device, model, sweep, lmax, batch=ni, grid=grid,
                            precision="tf32x3")
    seeds = [spectral_seed(lmax, sweep[k], 1 + k) for k in range(ni)]
    U0 = np.stack([q[0] for q in seeds])
    V0 = np.stack([q[1] for q in seeds])
    s.gpu.upload("U", U0)
    s.gpu.upload("V", V0)
    s.step(nsteps)
    U, V = s.read("U"), s.read("V")
    s.destroy()
    ref = O.ShtReference(lmax, lmax, *grid)
    for k in (0, 63):
        out = ref.model_step("schnakenberg", _prm("schnakenberg", sweep[k]),
                             np.stack([U0[k], V0[k]]).astype(np.float64), nsteps)
        for name, got, want, start in (("U", U[k], out[0], U0[k]), ("V", V[k], out[1], V0[k])):
            parity(f"schnakenberg lmax511 b64 4 steps inst{k} {name}", O.rel_l2(got, want),
                   TRANSFORM_BAR)
            parity(f"schnakenberg lmax511 b64 4 steps inst{k} d{name}",
                   O.rel_l2(got.astype(np.float64) - start, want - start), FIELD_BAR)
