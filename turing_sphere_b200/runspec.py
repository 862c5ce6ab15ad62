"""Run specifications of the solver benchmark: preset, lmax, seed, steps,
warmup and model parameters, parsed from and formatted back to a command
line (src/bench/runSpec.ts:36-135 of the reference: the same defaults, flag
grammar and error messages, so a command printed by one runs on the other
with only the program name changed)."""
from __future__ import annotations

import math
from dataclasses import dataclass, field

from .registry import defaultParams, mModelByKey, presets

RUN_COMMAND = "python -m turing_sphere_b200.run"
DEFAULT_LMAX = 63
DEFAULT_SEED = 1
DEFAULT_STEPS = 2000
DEFAULT_WARMUP = 100


@dataclass
class RunSpec:
    preset: str
    lmax: int = DEFAULT_LMAX
    seed: float = DEFAULT_SEED
    steps: int = DEFAULT_STEPS
    warmup: int = DEFAULT_WARMUP
    params: dict = field(default_factory=dict)

    def as_json(self) -> dict:
        seed = int(self.seed) if float(self.seed).is_integer() else self.seed
        return {"preset": self.preset, "lmax": self.lmax, "seed": seed, "steps": self.steps,
                "warmup": self.warmup, "params": dict(self.params)}


def resolvePreset(key: str):
    """(model, parameters) of a preset: the model's defaults overlaid with the
    preset's values (runSpec.ts:44-60)."""
    p = next((x for x in presets if x.key == key), None)
    if p is None:
        raise ValueError(f"unknown preset '{key}' (have: {', '.join(x.key for x in presets)})")
    model = mModelByKey(p.modelKey)
    if model is None:
        raise ValueError(f"preset '{key}' names unknown model '{p.modelKey}'")
    params = defaultParams(model)
    params.update(p.params)
    return model, params


def modelForSpec(spec: RunSpec):
    return resolvePreset(spec.preset)[0]


def _num(v: float) -> str:
    """JavaScript's String(number) for the values a spec holds."""
    if float(v).is_integer() and abs(v) < 1e21:
        return str(int(v))
    r = repr(float(v))
    if "e" in r:
        mant, ex = r.split("e")
        ex = int(ex)
        r = f"{mant}e{'+' if ex > 0 else '-'}{abs(ex)}"
    return r


def formatCommand(spec: RunSpec) -> str:
    """The command line that reproduces this run (runSpec.ts:74-86)."""
    model = modelForSpec(spec)
    parts = [RUN_COMMAND, f"--preset {spec.preset}", f"--lmax {spec.lmax}",
             f"--steps {spec.steps}", f"--seed {_num(spec.seed)}"]
    parts += [f"--{p.key} {_num(spec.params[p.key])}" for p in model.params]
    if spec.warmup != DEFAULT_WARMUP:
        parts.append(f"--warmup {spec.warmup}")
    return " ".join(parts)


def parseArgs(argv) -> RunSpec:
    """Inverse of formatCommand: `--key value` or `--key=value` in any order;
    ValueError with a usable message on anything unrecognised
    (runSpec.ts:90-135)."""
    flags = {}
    i = 0
    while i < len(argv):
        arg = argv[i]
        if not arg.startswith("--"):
            raise ValueError(f"unexpected argument '{arg}'")
        if "=" in arg:
            key, value = arg[2:].split("=", 1)
        else:
            key = arg[2:]
            i += 1
            value = argv[i] if i < len(argv) else None
        if value is None:
            raise ValueError(f"--{key} needs a value")
        if not key:
            raise ValueError(f"bad option '{arg}'")
        flags[key] = value
        i += 1

    def number(key, dflt):
        raw = flags.pop(key, None)
        if raw is None:
            return dflt
        try:
            v = float(raw)
        except ValueError:
            v = math.nan
        if not math.isfinite(v):
            raise ValueError(f"--{key} must be a number (got '{raw}')")
        return v

    def count(key, dflt, lo):
        v = number(key, dflt)
        if not float(v).is_integer() or v < lo:
            raise ValueError(f"--{key} must be an integer >= {lo} (got '{_num(v)}')")
        return int(v)

    preset = flags.pop("preset", presets[0].key)
    model, params = resolvePreset(preset)
    spec = RunSpec(preset=preset, lmax=count("lmax", DEFAULT_LMAX, 1),
                   seed=number("seed", DEFAULT_SEED), steps=count("steps", DEFAULT_STEPS, 1),
                   warmup=count("warmup", DEFAULT_WARMUP, 0), params=params)
    for p in model.params:
        raw = flags.pop(p.key, None)
        if raw is None:
            continue
        try:
            v = float(raw)
        except ValueError:
            v = math.nan
        if not math.isfinite(v):
            raise ValueError(f"--{p.key} must be a number (got '{raw}')")
        spec.params[p.key] = v
    if flags:
        raise ValueError(f"unknown option(s): {', '.join('--' + k for k in flags)}\n"
                         f"parameters of {model.label}: "
                         f"{' '.join('--' + p.key for p in model.params)}")
    return spec
