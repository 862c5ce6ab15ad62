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
    """--impl reference: the reference's CPU transform path, restated (oracle)."""
    rank = int(os.environ.get("RANK", "0"))
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
        "config": {"workload": f"SHT round trip, lmax {lmax}, {nlat}x{nphi} Gauss grid, "
                               f"{per_step} fields/step sample of the B={args.batch} batch"},
        "cpu_baseline": {"value": value, "unit": "SHT pairs/s", "cores": cores, "kind": "port",
                         "sample": f"{per_step} single-field pairs per step, f64 oracle "
                                   "(src/sht/reference.ts restated in C, OpenMP)"},
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


def time_e2e(plan, q0, qa, qb, spat, B, K, stream, world, dist):
    """End to end through the C ABI: every step copies its coefficients from
    pinned host memory, runs synth + analys and copies the result back.  The
    copies run on two copy streams (host->device and device->host, full duplex
    on PCIe) against double-buffered device arrays, so step i's transforms
    overlap step i+1's upload and step i-1's download, as a serving loop would
    run them.  Returns (ms for the timed steps, steps, relL2 of the last result)."""
    import torch
    hq_in = torch.from_numpy(q0).pin_memory()
    hq_out = [torch.empty_like(hq_in).pin_memory() for _ in range(2)]
    d_in = [qa, torch.empty_like(qa)]
    d_out = [qb, torch.empty_like(qb)]
    h2d, d2h = torch.cuda.Stream(), torch.cuda.Stream()
    sp = stream.cuda_stream
    Ke = max(3, K // 4)
    loaded = [torch.cuda.Event() for _ in range(2)]
    computed = [torch.cuda.Event() for _ in range(2)]
    saved = [torch.cuda.Event() for _ in range(2)]

    def run(n):
        for i in range(n):
            j = i & 1
            if i >= 2:
                h2d.wait_event(computed[j])        # step i-2 is done reading d_in[j]
            with torch.cuda.stream(h2d):
                d_in[j].copy_(hq_in, non_blocking=True)
                loaded[j].record(h2d)
            stream.wait_event(loaded[j])
            if i >= 2:
                stream.wait_event(saved[j])        # step i-2's result has left d_out[j]
            plan.synth_dev(d_in[j].data_ptr(), spat.data_ptr(), B, sp)
            plan.analys_dev(spat.data_ptr(), d_out[j].data_ptr(), B, sp)
            computed[j].record(stream)
            d2h.wait_event(computed[j])
            with torch.cuda.stream(d2h):
                hq_out[j].copy_(d_out[j], non_blocking=True)
                saved[j].record(d2h)
        stream.wait_stream(h2d)
        stream.wait_stream(d2h)

    run(3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    h2d.wait_event(e0)
    d2h.wait_event(e0)
    run(Ke)
    e1.record(stream)
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ems], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ems = float(t.item())
    back = hq_out[(Ke - 1) & 1].numpy()
    err = float(np.sqrt(((back - q0) ** 2).sum() / (q0 ** 2).sum()))
    return ems, Ke, err


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
    from turing_sphere_b200 import (GpuModel, ShtConfig, ShtPlan, defaultParams, mModelByKey,
                                    seededNoise)
    model = mModelByKey("brusselator")
    base = defaultParams(model)
    ni, npts = 256, 192 * 384
    rng = np.random.default_rng(3)
    sweep = []
    for _ in range(ni):
        a = rng.uniform(2.5, 3.5)
        lo = (1 + a * math.sqrt(base["D1"] / base["D2"])) ** 2
        sweep.append(dict(base, A=a, B=rng.uniform(lo, 1 + a * a)))
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


def main():
    args = parse()
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

    ems, Ke, e2e_err = time_e2e(plan, q0, qa, qb, spat, B, K, stream, world, dist)

    # IMEX steps: batched Schnakenberg instances on the same grid, both precisions
    del spat, fm
    torch.cuda.empty_cache()
    ni = args.imex_instances
    imex_tc_ms, imex_launches, ok_tc = time_imex(dev, plan, ni, args.imex_steps, 3, stream)
    imex_fp_ms, _, ok_fp = time_imex(dev, plain, ni, max(10, args.imex_steps // 4), 3, stream)
    c1_fp32 = time_imex_single_lmax63(dev, stream, "fp32")
    c1_tc = time_imex_single_lmax63(dev, stream, "tf32x3")
    c3 = time_brusselator_sweep(dev, stream)
    c3["ragged"] = time_ragged(dev, stream)
    a4_s, a4_ok = time_adjoint(dev, "allencahn", 255, 384, 768, 1, 256, 32)
    a5_s, a5_ok = time_adjoint(dev, "schnakenberg", 511, 768, 1536, 64, 64, 32)

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

        roof = stage_roofline(name, stage_ms[name], alg_bytes[name], leg_flop, passes, hbm, bf16,
                              of)
        roof["traffic"] = profiled_traffic(name)
        roof["traffic_source"] = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                  "launch (profiles/sht_pair_lmax255_b256_kernels.txt)")
        roof["stage_ms"] = stage_ms
        roof["stages"] = {
            st: {k: v for k, v in stage_roofline(st, stage_ms[st], alg_bytes[st], leg_flop, passes,
                                                 hbm, bf16, of).items()
                 if k in ("bound", "achieved", "unit", "frac")} for st in stages}
        cpu = cpu_baseline(lmax, nlat, nphi, budget_s=10.0, threads=0)
        one = cpu_baseline(lmax, nlat, nphi, budget_s=5.0, threads=1)
        cpu["single_thread"] = {k: one[k] for k in ("value", "cores", "sample")}
        cpu["other_configs"] = cpu_baselines_extra()
        line = {
            "metric": METRIC, "value": value, "unit": "SHT pairs/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": ms / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"batched SHT round trip (synth+analys), lmax=mmax={lmax}, "
                                   f"{nlat}x{nphi} Gauss grid, B={B} fields per GPU",
                       "precision": args.precision, "fourier": plan.fourierMode,
                       "fft_radices": plan.fftRadices, "kernel_shapes": plan.shapes,
                       "global_batch": B * world,
                       "l2": f"inputs larger than L2 (grid fields {sp_b / 1e6:.0f} MB/step)"},
            "e2e": {"value": world * B * Ke / (ems / 1e3), "unit": "SHT pairs/s",
                    "h2d_bytes_per_step": int(nlm_b), "d2h_bytes_per_step": int(nlm_b),
                    "round_trip_rel_l2": e2e_err},
            "gpu_launches": launches_per_pair(plan) * K,
            "plain_fp32": {"value": world * B * max(20, K // 4) / (plain_ms / 1e3),
                           "unit": "SHT pairs/s", "stage_ms": plain_stage},
            "imex": {"model": "schnakenberg (2 species), D1 sweep", "instances": ni,
                     "grid": f"lmax {lmax}, {nlat}x{nphi}", "launches_per_step": imex_launches,
                     "tc_steps_per_s": world * ni * args.imex_steps / (imex_tc_ms / 1e3),
                     "tc_steps_per_s_per_instance": args.imex_steps / (imex_tc_ms / 1e3),
                     "fp32_steps_per_s": world * ni * max(10, args.imex_steps // 4) / (imex_fp_ms / 1e3),
                     "unit": "instance-steps/s", "finite": ok_tc and ok_fp,
                     "single_lmax63": {"workload": "1 Schnakenberg instance, lmax 63, 96x192, "
                                             "2000 steps as captured step graphs",
                                 "fp32_steps_per_s": c1_fp32, "tc_steps_per_s": c1_tc}},
            "brusselator_sweep_lmax127": c3,
            "adjoint": {
                "allencahn_lmax255": {"workload": "Allen-Cahn, 1 instance, lmax 255, 384x768, tf32x3, "
                                        "256 steps forward + adjoint, checkpoints every 32",
                            "steps_per_s": 256 / a4_s, "finite": a4_ok},
                "schnakenberg_lmax511": {"workload": "Schnakenberg, 64 instances, lmax 511, 768x1536, "
                                        "tf32x3, 64 steps forward + adjoint, checkpoints every 32, "
                                        "gradients w.r.t. (a, b, D1, D2, dt) and the state",
                            "instance_steps_per_s": 64 * 64 / a5_s, "finite": a5_ok},
                "note": "wall-clock around ts_model_forward_backward (host round trips "
                        "of the cotangents included)"},
            "roofline": roof,
            "cpu_baseline": cpu,
            "clocks": sampler.summary(),
            "round_trip_rel_l2": rt,
            "flop_per_pair": flop_per_pair(lmax, lmax, nlat, nphi),
            "bytes_per_pair": bytes_per_pair(lmax, lmax, nlat, nphi),
        }
        line["imex"]["tc_vs_fp32"] = line["imex"]["tc_steps_per_s"] / line["imex"]["fp32_steps_per_s"]
        line["tc_vs_plain_sht"] = value / line["plain_fp32"]["value"]
        print(json.dumps(line), flush=True)
    return finish(plan, plain, dev, world)


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
