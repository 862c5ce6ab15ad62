"""Run digests for cross-environment comparison (src/mgpu/digest.ts)."""
from __future__ import annotations

import math

import numpy as np


def digestOf(values, fourier: str, adapter: str) -> dict:
    v = np.asarray(values, dtype=np.float64).ravel()
    return {"n": int(v.size), "min": float(v.min()), "max": float(v.max()),
            "mean": float(v.mean()), "rms": float(math.sqrt(float(np.mean(v * v)))),
            "fourier": fourier, "adapter": adapter}


def relL2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(math.sqrt(float(np.sum((a - b) ** 2)) / max(float(np.sum(b * b)), 1e-300)))


def formatDigest(d: dict) -> str:
    g = lambda v: f"{v:.9g}"  # noqa: E731
    return (f"n={d['n']} min={g(d['min'])} max={g(d['max'])} mean={g(d['mean'])} "
            f"rms={g(d['rms'])} fourier={d['fourier']}")


def digestDrift(a: dict, b: dict) -> float:
    def rel(x, y):
        return abs(x - y) / max(abs(x), abs(y), 1e-30)
    return max(rel(a[k], b[k]) for k in ("min", "max", "mean", "rms"))
