"""The available models and the metadata the host owns (src/mgpu/registry.ts).

A model's algorithm is its .m file (turing_sphere_b200/models/); its parameter
names, defaults and ranges, displayed species, dealiasing degree and seed
amplitude live here.  Spectral state names are the species names uppercased.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

HERE = os.path.dirname(os.path.abspath(__file__))


@dataclass(frozen=True)
class ParamSpec:
    key: str
    label: str
    value: float
    min: float
    max: float
    step: float


@dataclass
class MModel:
    key: str
    label: str
    blurb: str
    species: list
    state: list
    params: list
    pdeg: int
    seedAmp: float
    source: str = field(repr=False)


def _src(name: str) -> str:
    with open(os.path.join(HERE, "models", name)) as fh:
        return fh.read()


def _state(species):
    return [s.upper() for s in species]


schnakenberg = MModel(
    "schnakenberg", "Schnakenberg",
    "Turing spots; the homogeneous state is unstable to degrees 14 <= l <= 40, most strongly l = 24.",
    ["u", "v"], _state(["u", "v"]),
    [ParamSpec("a", "a", 0.1, 0.01, 0.5, 0.01), ParamSpec("b", "b", 0.9, 0.1, 2, 0.05),
     ParamSpec("D1", "D1", 4e-4, 1e-5, 5e-3, 1e-5), ParamSpec("D2", "D2", 8e-3, 1e-4, 5e-2, 1e-4),
     ParamSpec("dt", "dt", 0.05, 0.005, 0.5, 0.005)],
    3, 1e-2, _src("schnakenberg.m"))

brusselator = MModel(
    "brusselator", "Brusselator",
    "Turing stripes and spots from a smaller diffusivity contrast and a stiffer reaction.",
    ["u", "v"], _state(["u", "v"]),
    [ParamSpec("A", "A", 3, 0.5, 6, 0.1), ParamSpec("B", "B", 9, 1, 15, 0.25),
     ParamSpec("D1", "D1", 3.33e-3, 1e-4, 2e-2, 1e-4),
     ParamSpec("D2", "D2", 1.67e-2, 1e-3, 1e-1, 1e-3),
     ParamSpec("dt", "dt", 0.02, 0.002, 0.1, 0.002)],
    3, 1e-2, _src("brusselator.m"))

allencahn = MModel(
    "allencahn", "Allen-Cahn",
    "One species: interfaces form and coarsen until one domain swallows the sphere.",
    ["u"], _state(["u"]),
    [ParamSpec("eps2", "eps2", 1e-3, 1e-4, 1e-2, 1e-4), ParamSpec("dt", "dt", 0.02, 0.002, 0.2, 0.002)],
    3, 1e-2, _src("allencahn.m"))

mModels = [schnakenberg, brusselator, allencahn]


def mModelByKey(key: str):
    return next((m for m in mModels if m.key == key), None)


def defaultParams(m: MModel) -> dict:
    return {p.key: p.value for p in m.params}


@dataclass(frozen=True)
class Preset:
    key: str
    label: str
    modelKey: str
    params: dict = field(default_factory=dict)


presets = [
    Preset("schnak-spots", "Schnakenberg - spots", "schnakenberg"),
    Preset("schnak-coarse", "Schnakenberg - coarse spots", "schnakenberg", {"D1": 1e-3, "D2": 2e-2}),
    Preset("schnak-fine", "Schnakenberg - fine spots", "schnakenberg", {"D1": 1.6e-4, "D2": 3.2e-3}),
    Preset("brussel", "Brusselator - stripes & spots", "brusselator"),
    Preset("allencahn", "Allen-Cahn - coarsening", "allencahn"),
]


def brusselatorSweep(n: int, seed: int = 3, base: dict | None = None) -> list:
    """Parameter sets for a Brusselator sweep over its Turing-unstable band:
    A ~ U[2.5, 3.5], then B ~ U between the Turing threshold
    (1 + A sqrt(D1/D2))^2 and the Hopf bound 1 + A^2, with D1, D2 and dt the
    model's defaults (brusselator.m:22-28; registry.ts:79-83 of the
    reference).  Deterministic for a given seed."""
    import math

    import numpy as np

    p = dict(base or defaultParams(brusselator))
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        a = float(rng.uniform(2.5, 3.5))
        lo = (1 + a * math.sqrt(p["D1"] / p["D2"])) ** 2
        out.append(dict(p, A=a, B=float(rng.uniform(lo, 1 + a * a))))
    return out
