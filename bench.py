#!/usr/bin/env python
"""Benchmark of the spherical-harmonic transform hot path on B200.

Workload (one "step"): one synthesis + one analysis ("an SHT pair", the
reference's round trip, scripts/bench-sht.ts:7-9) of B = 256 real fields at
lmax = mmax = 255 on the 384 x 768 Gauss grid, coefficients seeded Gaussian
scaled by (l+1)^-1.  Spectral buffers ping-pong as in bench-sht.ts:160-205.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on rank 0.  ``value`` = SHT pairs/s over all ranks (inputs
resident in HBM); ``e2e`` = the same with the step's coefficients copied
host->device and the result device->host (pinned) inside the timed region.
``--impl reference`` times the CPU restatement of the reference's f64
transform (the reference itself is TypeScript/WebGPU and cannot run here) on
the host cores.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LMAX = 255
BATCH = 256
METRIC = "IMEX steps/s & SHT pairs/s @lmax255: TC+batched vs plain FP32, <=1e-5 vs f64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--lmax", type=int, default=LMAX)
    ap.add_argument("--batch", type=int, default=BATCH)
    ap.add_argument("--precision", default="tf32x3")
    ap.add_argument("--imex-instances", type=int, default=128)
    ap.add_argument("--imex-steps", type=int, default=100)
    ap.add_argument("--only", choices=["all", "sht", "imex"], default="all",
                    help="sht: the timed transform pairs alone; imex: the model steps alone "
                         "(short runs for a profiler's launch list)")
    ap.add_argument("--skip-single", action="store_true",
                    help="with --only imex: leave out the 2000-step single-instance lmax-63 runs")
    ap.add_argument("--no-autotune", action="store_true",
                    help="plans keep their default kernel shapes (no tuning launches, so a "
                         "profiler's launch skip count lands on the timed kernels)")
    return ap.parse_args()


def grid(lmax):
    nlat = (3 * (lmax + 1) + 1) // 2
    nlat += nlat & 1
    return nlat, 2 * nlat


def spectrum(lmax, seed):
    """Seeded Gaussian coefficients scaled by (l+1)^-1, m = 0 imaginary zero."""
    rng = np.random.default_rng(seed)
    q = rng.standard_normal((lmax + 1) * (lmax + 2)).astype(np.float32)
    l_of = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    m_of = np.concatenate([np.full(lmax + 1 - m, m) for m in range(lmax + 1)])
    q = q.reshape(-1, 2) / (l_of[:, None] + 1.0)
    q[m_of == 0, 1] = 0.0
    return np.ascontiguousarray(q.ravel(), dtype=np.float32)


class ClockSampler:
    """Samples SM clock and throttle reasons through NVML while running."""

    REASONS = {
        0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap",
        0x8: "hw_slowdown", 0x10: "sync_boost", 0x20: "sw_thermal_slowdown",
        0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown",
    }

    def __init__(self, index):
        self.samples, self.reasons, self.ok = [], 0, False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.max_mhz = None
        self._stop = threading.Event()

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM))
                self.reasons |= self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            except Exception:
                pass
            time.sleep(0.05)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["nvml unavailable"]}
        names = [n for b, n in self.REASONS.items() if self.reasons & b and n != "gpu_idle"]
        return {"sm_mhz": float(np.median(self.samples)), "sm_max_mhz": self.max_mhz,
                "reasons": names, "samples": len(self.samples)}


PROFILE = os.path.join(ROOT, "profiles", "sht_pair_lmax255_b256_kernels.txt")
STAGE_KERNELS = {"legSynth": ["ts_k_qimage", "ts_leg_synth_tc"], "fourSynth": ["ts_f2_synth"],
                 "fourAnalysW": ["ts_f2_analys_w"], "legAnalysW": ["ts_leg_analys_tc"],
                 "fourAnalys": ["ts_f2_analys<"], "legAnalys": ["ts_leg_analys"]}


def profiled_traffic(stage):
    """DRAM bytes (read + write) of one launch of the stage's kernels, from
    the committed ncu summary of this workload, or None."""
    if not os.path.exists(PROFILE):
        return None
    total, found = 0.0, False
    with open(PROFILE) as fh:
        for line in fh:
            if not line.startswith("kernel ") or "dram_read_MB" not in line:
                continue
            name = line[len("kernel "):line.index(" time_us")]
            if not any(name.startswith(k) for k in STAGE_KERNELS[stage]):
                continue
            f = line.split()
            total += (float(f[f.index("dram_read_MB") + 1]) +
                      float(f[f.index("dram_write_MB") + 1])) * 1e6
            found = True
    return total if found else None


def stage_roofline(stage, ms, alg_bytes, leg_flop, passes, hbm, bf16, of):
    """Roofline of one pair stage (ms per launch): the larger of its HBM floor
    (algorithmic bytes / bandwidth in GB/s) and, for a Legendre stage, its
    tensor floor (`passes` split-TF32 passes of `leg_flop` at the dense TF32
    rate bf16 / 2 TFLOP/s); `of` names the peaks' source."""
    dur = ms / 1e3
    t_hbm = alg_bytes / (hbm * 1e9)
    t_tc = passes * leg_flop / (bf16 / 2 * 1e12) if stage.startswith("leg") else 0.0
    if t_tc > t_hbm:
        return {"kernel": stage, "bound": "tensor", "achieved": leg_flop / dur / 1e12,
                "peak": bf16 / 2, "unit": "TFLOP/s", "frac": leg_flop / dur / 1e12 / (bf16 / 2),
                "peak_source": f"bf16_tflops / 2, the dense TF32 rate ({of})",
                "algorithmic_flop": leg_flop}
    r = {"kernel": stage, "bound": "hbm", "achieved": alg_bytes / dur / 1e9, "peak": hbm,
         "unit": "GB/s", "frac": alg_bytes / dur / 1e9 / hbm, "peak_source": f"hbm_gbs ({of})",
         "algorithmic_bytes": alg_bytes}
    if stage.startswith("leg"):
        r["tensor_floor_us"] = t_tc * 1e6
        r["hbm_floor_us"] = t_hbm * 1e6
        r["tensor_pipe_tflops"] = passes * leg_flop / dur / 1e12
        r["note"] = (f"HBM-bound: moving its inputs and outputs takes longer than its "
                     f"{passes} split-TF32 tensor passes at the dense TF32 rate")
    return r


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            p = json.load(fh)
        return p.get("hbm_gbs", 6650.0), p.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def cpu_baseline(lmax, nlat, nphi, budget_s=10.0, threads=0):
    """The f64 oracle transform on the host cores: SHT pairs/s on a bounded
    sample of the same workload (as many single-field pairs as fit the budget)."""
    from oracle import oracle as O
    ref = O.ShtReference(lmax, lmax, nlat, nphi, threads=threads)
    q = spectrum(lmax, 0).astype(np.float64)
    t0 = time.perf_counter()
    ref.analys(ref.synth(q))
    one = time.perf_counter() - t0
    n = max(1, min(200, int(budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    for i in range(n):
        q = ref.analys(ref.synth(q))
    dt = time.perf_counter() - t0
    cores = threads or os.cpu_count()
    return {"value": n / dt, "unit": "SHT pairs/s", "cores": cores, "kind": "port",
            "sample": f"{n} single-field pairs at lmax {lmax} ({nlat}x{nphi}), f64 direct "
                      f"summation (oracle restating src/sht/reference.ts), {dt:.1f} s"}


def cpu_baselines_extra():
    """The rest of the CPU baseline plan: SHT pairs/s at lmax 127 and 511 on
    one core and on all cores (bounded samples: 1-3 pairs at lmax 511), and
    Schnakenberg IMEX steps/s at lmax 63 (96x192) on one core, all by the f64
    oracle on the host."""
    from oracle import oracle as O
    out = {}
    for lm, budget in ((127, 2.0), (511, 3.0)):
        nlat, nphi = grid(lm)
        row = {}
        for key, th in (("all_cores", 0), ("single_thread", 1)):
            r = cpu_baseline(lm, nlat, nphi, budget_s=budget, threads=th)
            row[key] = {"value": r["value"], "cores": r["cores"], "sample": r["sample"]}
        out[f"sht_pairs_lmax{lm}"] = row
    ref = O.ShtReference(63, 63, 96, 192, threads=1)
    p = {"a": 0.1, "b": 0.9, "D1": 4e-4, "D2": 8e-3, "dt": 0.05}
    u00 = (p["a"] + p["b"]) * math.sqrt(4 * math.pi)
    st = np.zeros((2, 2 * ref.nlm))
    st[0, 0] = u00
    st[1, 0] = p["b"] / (p["a"] + p["b"]) ** 2 * math.sqrt(4 * math.pi)
    st += 1e-3 * np.random.default_rng(1).standard_normal(st.shape)
    prm = [p["a"], p["b"], p["D1"], p["D2"], p["dt"]]
    ref.model_step("schnakenberg", prm, st, 2)
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < 3.0:
        st = ref.model_step("schnakenberg", prm, st, 20)
        n += 20
    dt = time.perf_counter() - t0
    out["imex_schnakenberg_lmax63"] = {
        "value": n / dt, "unit": "steps/s", "cores": 1,
        "sample": f"{n} IMEX steps of one instance at lmax 63 (96x192), f64 oracle, {dt:.1f} s"}
    return out


def run_reference(args):
    """--impl reference: the reference's CPU transform path (src/sht/reference.ts,
    restated in C by the oracle: the reference itself is TypeScript on WebGPU
    and cannot run here) on all host cores, rank 0 only, on a bounded sample
    of this arm's workload: `per_step` single-field pairs per step."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    from oracle import oracle as O
    lmax = args.lmax
    nlat, nphi = grid(lmax)
    ref = O.ShtReference(lmax, lmax, nlat, nphi, threads=0)
    q = spectrum(lmax, 0).astype(np.float64)
    per_step = 2  # single-field pairs per step: a bounded sample of the batch
    for _ in range(args.warmup):
        q = ref.analys(ref.synth(q))
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for _ in range(per_step):
            q = ref.analys(ref.synth(q))
    dt = time.perf_counter() - t0
    value = per_step * args.steps / dt
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "SHT pairs/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(lmax, nlat, nphi, args.batch, world),
        "cpu_baseline": {"value": value, "unit": "SHT pairs/s", "cores": cores, "kind": "port",
                         "sample": f"{per_step} single-field pairs per step of the B={args.batch} "
                                   "batch, f64 oracle (src/sht/reference.ts restated in C, "
                                   "OpenMP over all host cores)"},
        "e2e": {"value": value, "unit": "SHT pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def time_pairs(plan, bufs, spat, B, K, W, stream):
    """K timed SHT pairs (W warm-up) through the public entry points
    ts_sht_synth_dev + ts_sht_analys_dev, spectral buffers ping-ponging as in
    bench-sht.ts:160-205; returns ms for the K pairs of batches."""
    import torch
    sp = stream.cuda_stream

    def step(i):
        src, dst = bufs[i & 1], bufs[(i + 1) & 1]
        plan.synth_dev(src.data_ptr(), spat.data_ptr(), B, sp)
        plan.analys_dev(spat.data_ptr(), dst.data_ptr(), B, sp)

    for i in range(W):
        step(i)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for i in range(K):
        step(i)
    t1.record(stream)
    torch.cuda.synchronize()
    plan.status()
    return t0.elapsed_time(t1)


def launches_per_pair(plan):
    """Kernels of one synth_dev + analys_dev: on a tensor-core plan the Q
    operand relayout, the tcgen05 synthesis, the two FFTs and the tcgen05
    analysis; on an FP32 plan two Legendre and two Fourier kernels."""
    return 5 if plan.wimageBytes(1) else 4


def stage_list(plan):
    """The kernels of one SHT pair as separately callable stages: on a
    tensor-core plan exactly those of synth_dev + analys_dev (the analysis
    writes the MMA operand image directly), else the four FP32 stages."""
    if plan.wimageBytes(1) and plan.fourierMode == "fft":
        return ["legSynth", "fourSynth", "fourAnalysW", "legAnalysW"]
    return ["legSynth", "fourSynth", "fourAnalys", "legAnalys"]


def time_stages(plan, bufs, spat, fm, B, K, W, stream):
    """Per-stage device time (CUDA events on the launching stream around each
    stage), averaged over K pairs after W warm-up; returns {stage: ms}."""
    import torch
    sp = stream.cuda_stream
    stages = stage_list(plan)
    wimg = None
    if stages[2] == "fourAnalysW":
        wimg = torch.zeros(plan.wimageBytes(B) // 4 + 1, dtype=torch.float32, device="cuda")
    mid = wimg if wimg is not None else fm

    def step(i, ev=None):
        src, dst = bufs[i & 1], bufs[(i + 1) & 1]
        ins = [src, fm, spat, mid]
        outs = [fm, spat, mid, dst]
        for k, st in enumerate(stages):
            if ev is not None:
                ev[k].record(stream)
            plan.stage_dev(st, ins[k].data_ptr(), outs[k].data_ptr(), B, sp)
        if ev is not None:
            ev[4].record(stream)

    for i in range(W):
        step(i)
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(K)]
    for i in range(K):
        step(i, evs[i])
    torch.cuda.synchronize()
    stage_ms = np.zeros(4)
    for e in evs:
        for k in range(4):
            stage_ms[k] += e[k].elapsed_time(e[k + 1])
    plan.status()
    return {s: float(v) / K for s, v in zip(stages, stage_ms)}


def time_imex(dev, plan, ninst, K, W, stream):
    """Schnakenberg, `ninst` instances with a parameter sweep of D1, advanced
    K steps (W warm-up) on `plan`'s grid; returns ms, launches per step and
    the spread of the final state (a sanity check that it ran)."""
    import torch
    from turing_sphere_b200 import GpuModel, defaultParams, mModelByKey, seededNoise
    model = mModelByKey("schnakenberg")
    p = defaultParams(model)
    gpu = GpuModel.create(dev, plan, model.source, [q.key for q in model.params], model.state,
                          model.species, ninst)
    gpu.setParams([dict(p, D1=p["D1"] * (1 + 0.5 * k / ninst)) for k in range(ninst)])
    npts = plan.cfg.nlat * plan.cfg.nphi
    gpu.init(np.concatenate([seededNoise(npts, model.seedAmp, 1 + k) for k in range(ninst)]))
    gpu.step(W)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    gpu.step(K)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    _, launches = gpu.counts("step")
    U = gpu.read("U")
    ok = bool(np.isfinite(U).all())
    gpu.destroy()
    plan.status()
    return ms, launches, ok


def time_e2e(plan, q0, B, K, world, dist):
    """End to end through the library's host-array round trip
    (ts_sht_roundtrip, the blocking call a reference-shaped host makes: host
    coefficients in, host coefficients out, the grid kept on the device): every
    step copies the batch's coefficients from page-locked host memory, runs
    synth + analys and copies the result back, the library pipelining the
    copies against the transforms over chunks of fields.  Host wall clock
    around the blocking calls, max over ranks.  Returns (ms for the timed
    steps, steps, relL2 of the last result)."""
    import torch
    hin = torch.from_numpy(np.ascontiguousarray(q0).ravel()).pin_memory()
    hout = torch.empty_like(hin).pin_memory()
    Ke = max(3, K // 4)
    for _ in range(2):  # grows the plan's staging arrays
        plan.roundtrip_ptr(hin.data_ptr(), hout.data_ptr(), B)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(Ke):
        plan.roundtrip_ptr(hin.data_ptr(), hout.data_ptr(), B)
    ems = (time.perf_counter() - t0) * 1e3
    if world > 1:
        t = torch.tensor([ems], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
    back = hout.numpy()
    ref = hin.numpy()
    err = float(np.sqrt(((back - ref) ** 2).sum() / (ref ** 2).sum()))
    return ems, Ke, err


def time_host_grid_pairs(plan, q0, B, K=3):
    """SHT pairs through the two host-array calls of the reference's ShtPlan
    (synth(Float32Array) -> grid on the host -> analys(Float32Array),
    sht.ts:414-461): the grid crosses PCIe both ways, 4.5x the bytes of the
    round trip.  Page-locked host arrays; host wall clock.  Returns pairs/s."""
    import torch
    nq, ns = q0.size, B * plan.cfg.nlat * plan.cfg.nphi
    hq = torch.from_numpy(np.ascontiguousarray(q0).ravel()).pin_memory()
    hs = torch.empty(ns, dtype=torch.float32).pin_memory()
    ho = torch.empty(nq, dtype=torch.float32).pin_memory()
    L, h = plan_lib(), plan.handle

    def step():
        chk(L.ts_sht_synth(h, ptr(hq), nq, ptr(hs), ns, B), plan)
        chk(L.ts_sht_analys(h, ptr(hs), ns, ptr(ho), nq, B), plan)

    step()
    t0 = time.perf_counter()
    for _ in range(K):
        step()
    return B * K / (time.perf_counter() - t0)


def plan_lib():
    from turing_sphere_b200 import _lib
    return _lib.lib()


def ptr(t):
    import ctypes as C
    return C.cast(t.data_ptr(), C.POINTER(C.c_float))


def chk(rc, plan):
    from turing_sphere_b200 import _lib
    _lib.check(rc, plan.device.handle)


def time_imex_single_lmax63(dev, stream, precision, K=2000, graphs=True):
    """A single Schnakenberg instance at lmax 63 on the 96 x 192 Gauss grid,
    K steps: the launch-latency-bound case, run as captured step graphs
    (default) or eager launches.  Returns steps/s."""
    import torch
    from turing_sphere_b200 import (GpuModel, ShtConfig, ShtPlan, defaultParams, mModelByKey,
                                    seededNoise)
    model = mModelByKey("schnakenberg")
    plan = ShtPlan.create(dev, ShtConfig(63, 63, 96, 192), {"precision": precision})
    gpu = GpuModel.create(dev, plan, model.source, [q.key for q in model.params], model.state,
                          model.species, 1)
    gpu.setGraphs(graphs)
    gpu.setParams(defaultParams(model))
    gpu.init(seededNoise(96 * 192, model.seedAmp, 1))
    gpu.step(10)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    gpu.step(K)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    gpu.destroy()
    plan.destroy()
    return K / (ms / 1e3)


def time_brusselator_sweep(dev, stream, K=200):
    """Brusselator parameter sweep: 256 instances with (A, B) spread over the
    Turing-unstable band, lmax 127 on 192 x 384, tensor-core plan, steps as
    captured graphs.  Returns instance-steps/s."""
    import torch
    from turing_sphere_b200 import GpuModel, ShtConfig, ShtPlan, mModelByKey, seededNoise
    from turing_sphere_b200.registry import brusselatorSweep
    model = mModelByKey("brusselator")
    ni, npts = 256, 192 * 384
    sweep = brusselatorSweep(ni, seed=3)
    plan = ShtPlan.create(dev, ShtConfig(127, 127, 192, 384), {"precision": "tf32x3",
                                                               "autotune": True})
    gpu = GpuModel.create(dev, plan, model.source, [q.key for q in model.params], model.state,
                          model.species, ni)
    gpu.setParams(sweep)
    gpu.init(np.concatenate([seededNoise(npts, model.seedAmp, 1 + k) for k in range(ni)]))
    gpu.step(5)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    gpu.step(K)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    finite = bool(np.isfinite(gpu.read("U")).all())
    gpu.destroy()
    plan.destroy()
    return {"workload": "Brusselator sweep, 256 instances, lmax 127, 192x384, tf32x3, "
                        f"{K} steps as captured step graphs",
            "instance_steps_per_s": ni * K / (ms / 1e3), "finite": finite}


def time_ragged(dev, stream, K=100):
    """The ragged sweep: 64 Brusselator instances at each of lmax
    63/127/255 (96x192, 192x384, 384x768 grids, one plan and model each),
    advanced as one model group (one captured graph per step, the three
    models on concurrent branches).  Returns instance-steps/s over all 192."""
    import torch
    from turing_sphere_b200 import (GpuModel, ModelGroup, ShtConfig, ShtPlan, defaultParams,
                                    mModelByKey, seededNoise)
    model = mModelByKey("brusselator")
    p = defaultParams(model)
    parts = []
    for lmax, nlat in ((63, 96), (127, 192), (255, 384)):
        plan = ShtPlan.create(dev, ShtConfig(lmax, lmax, nlat, 2 * nlat),
                              {"precision": "tf32x3", "autotune": True})
        gpu = GpuModel.create(dev, plan, model.source, [q.key for q in model.params],
                              model.state, model.species, 64)
        gpu.setParams(p)
        gpu.init(np.concatenate([seededNoise(nlat * 2 * nlat, model.seedAmp, 1 + k)
                                 for k in range(64)]))
        parts.append((plan, gpu))
    group = ModelGroup([g for _, g in parts])
    group.step(6)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    group.step(K)
    t1.record(stream)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    group.destroy()
    for plan, gpu in parts:
        gpu.destroy()
        plan.destroy()
    return {"workload": "Brusselator, 64 instances at each of lmax 63/127/255, one model "
                        f"group, {K} steps as captured group graphs",
            "instance_steps_per_s": 192 * K / (ms / 1e3)}


def time_adjoint(dev, key, lmax, nlat, nphi, ni, nsteps, every):
    """Forward + adjoint (ts_model_forward_backward) of `key` with `ni`
    instances: seconds for `nsteps` steps with checkpoints every `every`."""
    from turing_sphere_b200 import (GpuModel, ShtConfig, ShtPlan, defaultParams, mModelByKey,
                                    seededNoise)
    model = mModelByKey(key)
    plan = ShtPlan.create(dev, ShtConfig(lmax, lmax, nlat, nphi), {"precision": "tf32x3",
                                                                   "autotune": True})
    gpu = GpuModel.create(dev, plan, model.source, [q.key for q in model.params], model.state,
                          model.species, ni)
    gpu.setParams(defaultParams(model))
    gpu.init(np.concatenate([seededNoise(nlat * nphi, model.seedAmp, 1 + k) for k in range(ni)]))
    rng = np.random.default_rng(1)
    bar = {s: rng.standard_normal((ni, 2 * plan.nlm)).astype(np.float32) for s in model.state}
    # compiles the adjoint and grows every checkpoint and tape buffer the timed call needs
    gpu.forwardBackward(nsteps, every, bar)
    t0 = time.perf_counter()
    _, pbar = gpu.forwardBackward(nsteps, every, bar)
    dt = time.perf_counter() - t0
    ok = bool(np.isfinite(pbar).all())
    gpu.destroy()
    plan.destroy()
    return dt, ok


def launch_ranks(n):
    """`bench.py --gpus N` run without a launcher: start N ranks (one per GPU)
    under torch.distributed.run on 127.0.0.1 with the same arguments, and
    return their exit status.  Under a launcher (WORLD_SIZE set) it is not
    called."""
    import socket
    import subprocess
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args.gpus)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    from turing_sphere_b200 import ShtConfig, ShtPlan, Device
    from turing_sphere_b200.sht import bytes_per_pair, flop_per_pair

    lmax, B = args.lmax, args.batch
    nlat, nphi = grid(lmax)
    dev = Device(local)
    # a dedicated stream: torch's default current stream is the legacy NULL
    # stream, which the C ABI reads as "the context's own stream"
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    dev.set_stream(stream.cuda_stream)
    cfg = ShtConfig(lmax, lmax, nlat, nphi)
    tune = not args.no_autotune
    plan = ShtPlan.create(dev, cfg, {"precision": args.precision, "autotune": tune})
    plain = ShtPlan.create(dev, cfg, {"precision": "fp32", "autotune": tune})
    nlm = plan.nlm

    if args.only == "imex":
        ni = args.imex_instances
        ims, launches, ok = time_imex(dev, plan, ni, args.imex_steps, max(3, args.warmup), stream)
        c1 = {} if args.skip_single else {
            g: time_imex_single_lmax63(dev, stream, "fp32", graphs=g) for g in (True, False)}
        if rank == 0:
            print(json.dumps({"only": "imex", "instances": ni, "launches_per_step": launches,
                              "ms_per_step": ims / args.imex_steps, "finite": ok,
                              "value": world * ni * args.imex_steps / (ims / 1e3),
                              "unit": "instance-steps/s",
                              "single_lmax63_steps_per_s": {"graphs": c1.get(True),
                                                              "eager": c1.get(False)}}),
                  flush=True)
        return finish(plan, plain, dev, world)

    q0 = np.stack([spectrum(lmax, 1000 * rank + b) for b in range(B)])
    qa = torch.from_numpy(q0).cuda()
    qb = torch.empty_like(qa)
    spat = torch.empty(B, nlat * nphi, device="cuda")
    fm = torch.empty(B, 2 * (lmax + 1) * nlat, device="cuda")
    sp = stream.cuda_stream

    # correctness guard before timing (bench-sht.ts:252-318): one round trip
    plan.synth_dev(qa.data_ptr(), spat.data_ptr(), B, sp)
    plan.analys_dev(spat.data_ptr(), qb.data_ptr(), B, sp)
    torch.cuda.synchronize()
    plan.status()
    rt = float(torch.linalg.vector_norm(qb - qa) / torch.linalg.vector_norm(qa))
    if not math.isfinite(rt) or rt > 1e-3:
        print(json.dumps({"error": f"round trip relL2 {rt}"}), flush=True)
        return 1

    K, W = args.steps, max(3, args.warmup)
    # plain FP32 first (untimed by the clock sampler), then the headline path
    if args.only != "sht":
        Kp = max(20, K // 4)
        plain_ms = time_pairs(plain, [qa, qb], spat, B, Kp, W, stream)
        plain_stage = time_stages(plain, [qa, qb], spat, fm, B, Kp, W, stream)
    qa.copy_(torch.from_numpy(q0))
    sampler = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with sampler:
        ms = time_pairs(plan, [qa, qb], spat, B, K, W, stream)
    if world > 1:
        dist.barrier()
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    qa.copy_(torch.from_numpy(q0))
    stage_ms = time_stages(plan, [qa, qb], spat, fm, B, max(20, K // 4), W, stream)

    if args.only == "sht":
        if rank == 0:
            print(json.dumps({"only": "sht", "ms_per_step": ms / K, "stage_ms": stage_ms,
                              "kernel_shapes": plan.shapes,
                              "value": world * B * K / (ms / 1e3), "unit": "SHT pairs/s"}),
                  flush=True)
        return finish(plan, plain, dev, world)

    # free the transform buffers before the model workloads
    del spat, fm, qa, qb
    torch.cuda.empty_cache()
    ems, Ke, e2e_err = time_e2e(plan, q0, B, K, world, dist)
    host_grid = time_host_grid_pairs(plan, q0, B)

    # IMEX steps: batched Schnakenberg instances on the same grid, both precisions
    ni = args.imex_instances
    imex_tc_ms, imex_launches, ok_tc = time_imex(dev, plan, ni, args.imex_steps, 3, stream)
    kfp = max(10, args.imex_steps // 4)
    imex_fp_ms, _, ok_fp = time_imex(dev, plain, ni, kfp, 3, stream)
    c1_fp32 = time_imex_single_lmax63(dev, stream, "fp32")
    c1_tc = time_imex_single_lmax63(dev, stream, "tf32x3")
    c3 = time_brusselator_sweep(dev, stream, K=5000)
    c3["ragged"] = time_ragged(dev, stream, K=5000)
    a4_s, a4_ok = time_adjoint(dev, "allencahn", 255, 384, 768, 1, 1000, 32)
    a5_s, a5_ok = time_adjoint(dev, "schnakenberg", 511, 768, 1536, 64, 500, 32)
    c5 = time_forward_lmax511(dev, stream)

    if rank == 0:
        hbm, bf16, src = measured_peaks()
        pairs = world * B * K
        value = pairs / (ms / 1e3)
        stages = list(stage_ms)
        k = int(np.argmax([stage_ms[s] for s in stages]))
        name = stages[k]
        nlm_b = 8.0 * nlm * B
        fm_b = 8.0 * (lmax + 1) * nlat * B  # fm, G and the W image are all this size
        sp_b = 4.0 * nlat * nphi * B
        alg_bytes = {"legSynth": nlm_b + fm_b, "fourSynth": fm_b + sp_b,
                     "fourAnalys": sp_b + fm_b, "fourAnalysW": sp_b + fm_b,
                     "legAnalys": fm_b + nlm_b, "legAnalysW": fm_b + nlm_b}
        leg_flop = 2.0 * nlm * nlat * B  # complex x real FMA per (l, m, latitude pair)
        passes = 3 if args.precision != "fp32" else 1
        of = "of measured" if src == "measured" else "of fallback"

        roof = pair_roofline(ms / K, B, bytes_per_pair(lmax, lmax, nlat, nphi), hbm, of)
        roof["traffic"] = profiled_pair_traffic(stages)
        roof["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum, summed over "
                                  "the pair's kernels, one launch each "
                                  "(profiles/sht_pair_lmax255_b256_kernels.txt)")
        dom = stage_roofline(name, stage_ms[name], alg_bytes[name], leg_flop, passes, hbm, bf16,
                             of)
        dom["traffic"] = profiled_traffic(name)
        roof["dominant_kernel"] = dom
        roof["stage_ms"] = stage_ms
        roof["stages"] = {
            st: {k: v for k, v in stage_roofline(st, stage_ms[st], alg_bytes[st], leg_flop, passes,
                                                 hbm, bf16, of).items()
                 if k in ("bound", "achieved", "unit", "frac")} for st in stages}
        cpu = cpu_baseline(lmax, nlat, nphi, budget_s=10.0, threads=0)
        one = cpu_baseline(lmax, nlat, nphi, budget_s=5.0, threads=1)
        cpu["single_thread"] = {k: one[k] for k in ("value", "cores", "sample")}
        cpu["other_configs"] = cpu_baselines_extra()
        tc_imex = world * ni * args.imex_steps / (imex_tc_ms / 1e3)
        fp_imex = world * ni * kfp / (imex_fp_ms / 1e3)
        plain_pairs = world * B * max(20, K // 4) / (plain_ms / 1e3)
        line = {
            "metric": METRIC, "value": value, "unit": "SHT pairs/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": workload_config(lmax, nlat, nphi, B, world),
            "plan": {"precision": args.precision, "fourier": plan.fourierMode,
                     "fft_radices": plan.fftRadices, "kernel_shapes": plan.shapes},
            "e2e": {"value": world * B * Ke / (ems / 1e3), "unit": "SHT pairs/s",
                    "h2d_bytes_per_step": int(nlm_b), "d2h_bytes_per_step": int(nlm_b),
                    "path": "ts_sht_roundtrip (host coefficients in and out, page-locked; "
                            "copies pipelined by the library over chunks of fields; host wall "
                            "clock around the blocking calls)",
                    "round_trip_rel_l2": e2e_err,
                    "host_grid_pairs_per_s": host_grid,
                    "host_grid_path": "ts_sht_synth + ts_sht_analys with the grid on the host "
                                      "(sht.ts:414-461 shape: 4.5x the PCIe bytes)"},
            "gpu_launches": launches_per_pair(plan) * K,
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": sampler.summary(),
            "plain_fp32": {"value": plain_pairs, "unit": "SHT pairs/s", "stage_ms": plain_stage},
            "brusselator_sweep_lmax127": c3,
            "adjoint": {
                "allencahn_lmax255": {"workload": "Allen-Cahn, 1 instance, lmax 255, 384x768, tf32x3, "
                                        "1000 steps forward + adjoint, checkpoints every 32",
                            "steps_per_s": 1000 / a4_s, "finite": a4_ok},
                "schnakenberg_lmax511": {"workload": "Schnakenberg, 64 instances, lmax 511, 768x1536, "
                                        "tf32x3, 500 steps forward + adjoint, checkpoints every 32, "
                                        "gradients w.r.t. (a, b, D1, D2, dt) and the state",
                            "instance_steps_per_s": 64 * 500 / a5_s, "finite": a5_ok},
                "note": "wall-clock around ts_model_forward_backward (host round trips "
                        "of the cotangents included)"},
            "schnakenberg_lmax511_forward": c5,
            "round_trip_rel_l2": rt,
            "flop_per_pair": flop_per_pair(lmax, lmax, nlat, nphi),
            "bytes_per_pair": bytes_per_pair(lmax, lmax, nlat, nphi),
            # the metric's IMEX half and both ratios last, where a tail of the line shows them
            "imex": {"model": "schnakenberg (2 species), D1 sweep", "instances": ni,
                     "grid": f"lmax {lmax}, {nlat}x{nphi}", "launches_per_step": imex_launches,
                     "single_lmax63": {"workload": "1 Schnakenberg instance, lmax 63, 96x192, "
                                             "2000 steps as captured step graphs",
                                 "fp32_steps_per_s": c1_fp32, "tc_steps_per_s": c1_tc},
                     "finite": ok_tc and ok_fp,
                     "tc_ms_per_step": imex_tc_ms / args.imex_steps,
                     "fp32_ms_per_step": imex_fp_ms / kfp,
                     "tc_steps_per_s_per_instance": args.imex_steps / (imex_tc_ms / 1e3),
                     "unit": "instance-steps/s",
                     "tc_steps_per_s": tc_imex, "fp32_steps_per_s": fp_imex,
                     "tc_vs_fp32": tc_imex / fp_imex},
            "sht_pairs": {"tc_pairs_per_s": value, "fp32_pairs_per_s": plain_pairs,
                          "tc_vs_fp32": value / plain_pairs},
            "imex_tc_vs_fp32": tc_imex / fp_imex,
        }
        print(json.dumps(line), flush=True)
    return finish(plan, plain, dev, world)


def workload_config(lmax, nlat, nphi, B, world):
    """The `config` object, the same in both arms' lines."""
    return {"workload": f"batched SHT round trip (synth+analys), lmax=mmax={lmax}, "
                        f"{nlat}x{nphi} Gauss grid, B={B} fields per GPU",
            "global_batch": B * world,
            "l2": f"inputs larger than L2 (grid fields {4.0 * nlat * nphi * B / 1e6:.0f} MB/step)"}


def pair_roofline(ms_per_step, B, bytes_pair, hbm, of):
    """Roofline of the whole SHT pair: the minimum HBM bytes of one synth +
    one analys per field (coefficients and grid, read and written, both
    directions: 2 (8 nlm + 4 nlat nphi)) times the batch, over the device
    time of one pair of batches."""
    alg = bytes_pair * B
    ach = alg / (ms_per_step / 1e3) / 1e9
    return {"kernel": "SHT pair: all kernels of synth_dev + analys_dev", "bound": "hbm",
            "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
            "peak_source": f"hbm_gbs ({of})", "algorithmic_bytes": alg}


def profiled_pair_traffic(stages):
    """DRAM bytes of one SHT pair (every stage's kernels, one launch each)
    from the committed ncu summary, or None if a stage is missing."""
    total = 0.0
    for st in stages:
        t = profiled_traffic(st)
        if t is None:
            return None
        total += t
    return total


def time_forward_lmax511(dev, stream, ni=64, K=20):
    """The lmax-511 inverse-problem workload's forward step (64 Schnakenberg
    instances, 768 x 1536) on the tensor-core and on the plain FP32 plan
    (CUDA events, K steps each), with each plan's synthesis error against the
    f64 oracle on one seeded field: the comparison at the stated error."""
    from oracle import oracle as O
    from turing_sphere_b200 import ShtConfig, ShtPlan
    lmax, nlat, nphi = 511, 768, 1536
    out = {"workload": f"Schnakenberg, {ni} instances, lmax {lmax}, {nlat}x{nphi}, forward "
                       f"IMEX steps ({K} timed per plan)"}
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    q = spectrum(lmax, 5)
    want = ref.synth(q.astype(np.float64))
    for prec in ("tf32x3", "fp32"):
        plan = ShtPlan.create(dev, ShtConfig(lmax, lmax, nlat, nphi), {"precision": prec})
        ms, launches, ok = time_imex(dev, plan, ni, K, 3, stream)
        out[prec] = {"instance_steps_per_s": ni * K / (ms / 1e3), "ms_per_step": ms / K,
                     "launches_per_step": launches, "finite": ok,
                     "synth_rel_l2_vs_f64": float(np.sqrt(((plan.synth(q) - want) ** 2).sum()
                                                          / (want ** 2).sum()))}
        plan.destroy()
    out["tc_vs_fp32"] = out["tf32x3"]["instance_steps_per_s"] / out["fp32"]["instance_steps_per_s"]
    prof = profiled_kernels(PROFILE_511)
    if prof:
        out["ncu"] = prof
    return out


PROFILE_511 = os.path.join(ROOT, "profiles", "imex_schnakenberg_lmax511_i16_kernels.txt")


def profiled_kernels(path):
    """Per-kernel DRAM GB/s and tensor-pipe activity from a committed ncu
    summary (lines 'kernel <name> time_us T ... dram_gbs G ... tensor_pct P'),
    or None when the summary is absent."""
    if not os.path.exists(path):
        return None
    out = {}
    with open(path) as fh:
        for line in fh:
            if not line.startswith("kernel "):
                continue
            name = line[len("kernel "):line.index(" time_us")]
            f = line.split()
            row = {}
            for key in ("time_us", "dram_gbs", "tensor_pct"):
                if key in f:
                    row[key] = float(f[f.index(key) + 1])
            out[name.split("(")[0]] = row
    return {"source": os.path.relpath(path, ROOT), "kernels": out}


def finish(plan, plain, dev, world):
    plan.destroy()
    plain.destroy()
    dev.destroy()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
