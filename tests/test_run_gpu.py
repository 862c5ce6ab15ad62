"""The solver-benchmark runner (scripts/bench.ts of the reference) end to end
on a small grid: the --json object's shape, the dump file and its digest, and
that a second run from the same spec reproduces the digest bit for bit."""
import json
import subprocess
import sys

import numpy as np
import pytest

from turing_sphere_b200.digest import digestOf
from turing_sphere_b200.layout import gridForLmax
from turing_sphere_b200.registry import mModelByKey
from turing_sphere_b200.runspec import parseArgs

pytestmark = pytest.mark.gpu


def _run(args):
    out = subprocess.run([sys.executable, "-m", "turing_sphere_b200.run", *args],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    return out.stdout


def test_json_and_dump(tmp_path):
    dump = tmp_path / "state.json"
    args = ["--preset", "schnak-spots", "--lmax", "31", "--steps", "40", "--warmup", "3",
            "--seed", "5", "--batch", "8", "--json", "--dump-state", str(dump)]
    j = json.loads(_run(args))
    assert list(j) == ["command", "spec", "model", "backend", "grid", "compiled", "digest",
                       "throughput", "latency", "state"]
    nlat, nphi = gridForLmax(31, mModelByKey(j["model"]).pdeg)
    assert j["grid"] == {"lmax": 31, "nlat": nlat, "nphi": nphi, "nlm": 32 * 33 // 2}
    assert j["compiled"]["opsPerStep"] >= 1 and j["compiled"]["kernels"] >= 1
    assert j["throughput"]["batch"] == 8 and j["throughput"]["msPerStep"] > 0
    assert j["latency"]["minMs"] <= j["latency"]["medianMs"] <= j["latency"]["p95Ms"]
    # as in the reference, the digest run re-seeds, so the state reported is after --steps
    assert j["state"]["finite"] and j["state"]["steps"] == 40
    # the command it prints parses back to the same spec
    assert parseArgs(j["command"].split()[3:]).as_json() == j["spec"]
    d = json.loads(dump.read_text())
    assert d["digest"] == j["digest"] and d["command"] == j["command"]
    st = np.asarray(d["state"], dtype=np.float32)
    assert st.size == 2 * j["grid"]["nlm"]
    assert digestOf(st, j["digest"]["fourier"], j["digest"]["adapter"]) == d["digest"]
    again = json.loads(_run(args))
    assert again["digest"] == j["digest"]


def test_text_output():
    out = _run(["--preset", "allencahn", "--lmax", "15", "--steps", "10", "--warmup", "0",
                "--digest"])
    assert "ms/step" in out and "state after 10 steps from seed 1:" in out and "n=" in out


def test_bad_option_exits_2():
    out = subprocess.run([sys.executable, "-m", "turing_sphere_b200.run", "--nope", "1"],
                         capture_output=True, text=True, timeout=60)
    assert out.returncode == 2 and "unknown option(s): --nope" in out.stderr


def test_dump_matches_oracle_dump(tmp_path):
    """compare-native --check: the runner's dump of one spec against a dump of
    the same spec stepped by the f64 oracle from the same seeded initial state,
    diffed by the compare tool at the reference's 2e-3 relative L2."""
    from oracle import oracle as O
    from turing_sphere_b200 import compare
    from turing_sphere_b200.model import ModelSession
    from turing_sphere_b200.runspec import resolvePreset
    from turing_sphere_b200.sht import requestShtDevice

    gpu_dump = tmp_path / "gpu.json"
    args = ["--preset", "schnak-spots", "--lmax", "31", "--steps", "200", "--warmup", "0",
            "--seed", "3", "--dump-state", str(gpu_dump)]
    _run(args)
    spec = parseArgs(args[:-2])
    model, params = resolvePreset(spec.preset)
    s = ModelSession.create(requestShtDevice(0), model, spec.params, spec.lmax)
    s.seed(int(spec.seed))
    init = np.stack([s.read(k) for k in model.state]).astype(np.float64)
    cfg = s.cfg
    s.destroy()
    ref = O.ShtReference(cfg.lmax, cfg.mmax, cfg.nlat, cfg.nphi)
    out = ref.model_step(model.key, [spec.params[p.key] for p in model.params], init, spec.steps)
    state = out[0].astype(np.float32)
    ref_dump = tmp_path / "oracle.json"
    ref_dump.write_text(json.dumps({"command": "", "spec": spec.as_json(),
                                    "digest": digestOf(state, "fft", "f64 oracle"),
                                    "state": [float(v) for v in state]}))
    assert compare.main([str(gpu_dump), str(ref_dump)]) == 0
    r = compare.compare(compare.load(str(gpu_dump)), compare.load(str(ref_dump)))
    assert r["relL2"] < 1e-4, r
