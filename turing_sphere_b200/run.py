"""The solver benchmark of the reference (scripts/bench.ts) on this library:

  python -m turing_sphere_b200.run --preset schnak-spots --lmax 63 --steps 2000 --seed 1 \\
      --a 0.1 --b 0.9 --D1 0.0004 --D2 0.008 --dt 0.05 [--json] [--dump-state f]

Same options, the same two numbers (throughput: batches of steps awaited
once each; latency: one step per wait) and the same machine-readable shapes:
--json prints the object bench.ts prints (command, spec, model, backend,
grid, compiled, digest, throughput, latency, state) and --dump-state writes
{command, spec, digest, state}, the file scripts/compare-native.mjs and
compare-env.mjs diff against a WebGPU or native run.  --precision picks the
Legendre stage (fp32, the reference's arithmetic, or tf32x3).
"""
from __future__ import annotations

import json
import sys
import time

import numpy as np

from .runspec import (DEFAULT_LMAX, DEFAULT_SEED, DEFAULT_STEPS, DEFAULT_WARMUP, RUN_COMMAND,
                      _num, formatCommand, modelForSpec, parseArgs, presets)

USAGE = f"""usage: {RUN_COMMAND} [options]

  --preset <key>    {' | '.join(p.key for p in presets)}
                    (default {presets[0].key})
  --lmax <n>        spherical harmonic truncation (default {DEFAULT_LMAX})
  --steps <n>       timed steps (default {DEFAULT_STEPS})
  --warmup <n>      untimed steps first (default {DEFAULT_WARMUP})
  --seed <n>        initial-noise seed (default {DEFAULT_SEED})
  --batch <n>       steps per wait for the throughput number (default 16)
  --precision <p>   fp32 | tf32x3 (default fp32)
  --digest          after timing, re-run exactly --steps steps from the seed and
                      print a digest of the final state
  --dump-state <f>  like --digest, and write the state to <f> as JSON
  --<param> <v>     any parameter of the preset's model, e.g. --dt 0.05
  --json            machine-readable output
  --help"""


def timing(samples) -> dict:
    """bench.ts's latency summary of per-step wall times (ms)."""
    s = np.sort(np.asarray(samples, dtype=np.float64))
    q = lambda p: float(s[min(len(s) - 1, int(np.floor(p * len(s))))])
    total = float(s.sum())
    return {"meanMs": total / len(s), "medianMs": q(0.5), "p05Ms": q(0.05), "p95Ms": q(0.95),
            "minMs": float(s[0]), "totalMs": total, "stepsPerSec": 1000.0 * len(s) / total}


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    if "--help" in argv or "-h" in argv:
        print(USAGE)
        return 0
    want_json = "--json" in argv
    want_digest, dump, batch, precision, rest = False, None, 16, "fp32", []
    i = 0
    while i < len(argv):
        a = argv[i]
        if a == "--json":
            pass
        elif a == "--digest":
            want_digest = True
        elif a in ("--batch", "--dump-state", "--precision") or a.startswith(
                ("--batch=", "--dump-state=", "--precision=")):
            key, val = (a.split("=", 1) if "=" in a else (a, argv[i + 1] if i + 1 < len(argv) else None))
            if "=" not in a:
                i += 1
            if val is None:
                print(f"run: {key} needs a value", file=sys.stderr)
                return 2
            if key == "--batch":
                batch = int(val)
            elif key == "--dump-state":
                dump, want_digest = val, True
            else:
                precision = val
        else:
            rest.append(a)
        i += 1
    if batch < 1:
        print("run: --batch must be an integer >= 1", file=sys.stderr)
        return 2
    try:
        spec = parseArgs(rest)
    except ValueError as e:
        print(f"run: {e}\n\n{USAGE}", file=sys.stderr)
        return 2

    from .digest import digestOf, formatDigest
    from .model import ModelSession
    from .sht import requestShtDevice
    model = modelForSpec(spec)
    device = requestShtDevice(0)
    session = ModelSession.create(device, model, spec.params, spec.lmax, precision=precision)
    session.seed(int(spec.seed))
    kernels, launches = session.gpu.counts("step")
    cfg = session.cfg
    adapter = device.name

    session.step(spec.warmup)
    session.sync()
    runs, steps_run, t0 = 0, 0, time.perf_counter()
    encode = 0.0
    while steps_run < spec.steps:
        n = min(batch, spec.steps - steps_run)
        e0 = time.perf_counter()
        session.step(n)
        encode += time.perf_counter() - e0
        session.sync()
        steps_run += n
        runs += 1
    throughput_ms = (time.perf_counter() - t0) * 1e3 / steps_run
    samples = []
    for _ in range(min(spec.steps, 200)):
        s0 = time.perf_counter()
        session.step(1)
        session.sync()
        samples.append((time.perf_counter() - s0) * 1e3)
    lat = timing(samples)
    field = session.read(model.species[0])
    finite = bool(np.isfinite(field).all())

    digest, state = None, None
    if want_digest:
        session.seed(int(spec.seed))
        session.step(spec.steps)
        session.sync()
        state = session.read(model.state[0])
        digest = digestOf(state, session.sht.fourierMode, adapter)

    command = formatCommand(spec)
    if want_json:
        print(json.dumps({
            "command": command,
            "spec": spec.as_json(),
            "model": model.key,
            "backend": {"adapter": adapter, "runtime": "cuda, sm_100a",
                        "precision": precision},
            "grid": {"lmax": cfg.lmax, "nlat": cfg.nlat, "nphi": cfg.nphi,
                     "nlm": session.sht.nlm},
            "compiled": {"opsPerStep": launches, "kernels": kernels},
            "digest": digest,
            "throughput": {"batch": batch, "msPerStep": throughput_ms,
                           "stepsPerSec": 1000.0 / throughput_ms,
                           "encodeMsPerStep": encode * 1e3 / steps_run},
            "latency": lat,
            "state": {"t": session.t, "steps": session.steps, "species": model.species[0],
                      "min": float(field.min()), "max": float(field.max()),
                      "contrast": float(field.max() - field.min()), "finite": finite},
        }, indent=2))
    else:
        print(f"  {throughput_ms:.3f} ms/step   {1000 / throughput_ms:.1f} steps/s   "
              f"(batches of {batch})")
        print(f"  one step per wait: {lat['meanMs']:.3f} ms mean · median {lat['medianMs']:.3f}"
              f" · p05 {lat['p05Ms']:.3f} · p95 {lat['p95Ms']:.3f} · min {lat['minMs']:.3f}")
        print(f"  after {session.steps} steps: t = {session.t:.2f}, {model.species[0]} in "
              f"[{field.min():.4f}, {field.max():.4f}] (contrast {field.max() - field.min():.4f})"
              + ("" if finite else "  - NOT FINITE"))
        if digest:
            print(f"\n  state after {spec.steps} steps from seed {_num(spec.seed)}:")
            print(f"    {formatDigest(digest)}")
    if dump and state is not None and digest is not None:
        with open(dump, "w") as fh:
            json.dump({"command": command, "spec": spec.as_json(), "digest": digest,
                       "state": [float(v) for v in state]}, fh)
    return 0 if finite else 1


if __name__ == "__main__":
    sys.exit(main())
