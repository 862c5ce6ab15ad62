"""The run-spec grammar of the solver benchmark (src/bench/runSpec.ts:36-135):
defaults, --key value / --key=value, preset parameters, the command line a
spec formats to, and the error messages."""
import pytest

from turing_sphere_b200.runspec import (DEFAULT_LMAX, DEFAULT_STEPS, DEFAULT_WARMUP, RunSpec,
                                        formatCommand, parseArgs, resolvePreset)


def test_defaults_and_preset_parameters():
    s = parseArgs([])
    assert (s.preset, s.lmax, s.steps, s.warmup, s.seed) == ("schnak-spots", DEFAULT_LMAX,
                                                             DEFAULT_STEPS, DEFAULT_WARMUP, 1)
    assert s.params["a"] == 0.1 and s.params["D1"] == 4e-4
    s = parseArgs(["--preset", "schnak-coarse"])
    assert s.params["D1"] == 1e-3 and s.params["D2"] == 2e-2


def test_format_then_parse_round_trip():
    s = parseArgs(["--preset=brussel", "--lmax", "127", "--steps=50", "--seed", "7",
                   "--A", "3.1", "--warmup", "5"])
    cmd = formatCommand(s)
    assert cmd.startswith("python -m turing_sphere_b200.run --preset brussel --lmax 127 --steps 50 "
                          "--seed 7 --A 3.1 --B 9 --D1")
    assert cmd.endswith("--warmup 5")
    again = parseArgs(cmd.split()[3:])
    assert again == s


@pytest.mark.parametrize("argv,msg", [
    (["lmax"], "unexpected argument 'lmax'"),
    (["--lmax"], "--lmax needs a value"),
    (["--lmax", "0"], "--lmax must be an integer >= 1"),
    (["--steps", "2.5"], "--steps must be an integer >= 1"),
    (["--dt", "fast"], "--dt must be a number (got 'fast')"),
    (["--preset", "nope"], "unknown preset 'nope'"),
    (["--zz", "1"], "unknown option(s): --zz"),
])
def test_errors(argv, msg):
    with pytest.raises(ValueError, match=None) as e:
        parseArgs(argv)
    assert msg in str(e.value)


def test_spec_json_shape():
    s = parseArgs(["--preset", "allencahn", "--steps", "3"])
    j = s.as_json()
    assert list(j) == ["preset", "lmax", "seed", "steps", "warmup", "params"]
    assert j["params"] == resolvePreset("allencahn")[1]


def test_compare_dump_files(tmp_path):
    """The --check diff of two dump files: same spec and close states pass,
    a changed parameter or a perturbed state fails."""
    import json

    import numpy as np

    from turing_sphere_b200 import compare
    from turing_sphere_b200.digest import digestOf

    spec = parseArgs(["--lmax", "7", "--steps", "5"]).as_json()
    st = np.random.default_rng(0).standard_normal(72).astype(np.float32)

    def dump(name, state, sp=spec):
        p = tmp_path / name
        p.write_text(json.dumps({"command": "", "spec": sp, "state": [float(v) for v in state],
                                 "digest": digestOf(state, "fft", "x")}))
        return str(p)

    a = dump("a.json", st)
    assert compare.main([a, dump("b.json", st * (1 + 1e-5))]) == 0
    assert compare.main([a, dump("c.json", st + 0.1)]) == 1
    other = dict(spec, params=dict(spec["params"], dt=0.01))
    assert compare.main([a, dump("d.json", st, other)]) == 1
    assert compare.main([a]) == 2
