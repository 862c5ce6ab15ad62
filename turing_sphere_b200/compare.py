"""Diff two --dump-state files of the same spec (the --check half of the
reference's scripts/compare-native.mjs and compare-env.mjs):

  python -m turing_sphere_b200.compare a.json b.json [--tolerance 2e-3]

The files are the runner's wire format {command, spec, digest, state}.  Two
runs of one spec (preset, lmax, seed, steps, parameters) compute the same
thing up to fp32 round-off, so their final spectral states agree to a small
relative L2; exit 1 when the specs differ or the states are further apart
than the tolerance (2e-3, the reference's default)."""
from __future__ import annotations

import json
import sys

from .digest import digestDrift, formatDigest, relL2

DEFAULT_TOLERANCE = 2e-3


def load(path: str) -> dict:
    with open(path) as fh:
        d = json.load(fh)
    for k in ("spec", "digest", "state"):
        if k not in d:
            raise ValueError(f"{path}: not a --dump-state file (no '{k}')")
    return d


def spec_mismatch(a: dict, b: dict) -> list:
    """Spec keys that differ; warmup is not one (the reproducible state is
    exactly --steps steps from the seed, whatever was timed before it)."""
    keys = ("preset", "lmax", "seed", "steps")
    out = [k for k in keys if a.get(k) != b.get(k)]
    pa, pb = a.get("params", {}), b.get("params", {})
    out += [f"params.{k}" for k in sorted(set(pa) | set(pb)) if pa.get(k) != pb.get(k)]
    return out


def compare(a: dict, b: dict, tolerance: float = DEFAULT_TOLERANCE) -> dict:
    mismatch = spec_mismatch(a["spec"], b["spec"])
    if len(a["state"]) != len(b["state"]):
        mismatch.append("state length")
    rel = None if mismatch else relL2(a["state"], b["state"])
    return {"mismatch": mismatch, "relL2": rel,
            "digestDrift": digestDrift(a["digest"], b["digest"]),
            "ok": not mismatch and rel < tolerance}


def main(argv=None) -> int:
    argv = list(sys.argv[1:] if argv is None else argv)
    tol = DEFAULT_TOLERANCE
    if "--tolerance" in argv:
        i = argv.index("--tolerance")
        tol = float(argv[i + 1])
        del argv[i:i + 2]
    if len(argv) != 2:
        print("usage: python -m turing_sphere_b200.compare a.json b.json [--tolerance x]",
              file=sys.stderr)
        return 2
    a, b = load(argv[0]), load(argv[1])
    r = compare(a, b, tol)
    for path, d in zip(argv, (a, b)):
        print(f"  {path}: {formatDigest(d['digest'])} adapter={d['digest'].get('adapter')}")
    if r["mismatch"]:
        print(f"  different specs: {', '.join(r['mismatch'])}")
        return 1
    print(f"  relative L2 {r['relL2']:.3e} (tolerance {tol:.1e}), digest drift "
          f"{r['digestDrift']:.3e}: {'same computation' if r['ok'] else 'DIFFERENT'}")
    return 0 if r["ok"] else 1


if __name__ == "__main__":
    sys.exit(main())
