"""The C ABI library loads and exports every symbol its header declares.
No compute calls: this runs without a GPU."""
import os
import re

import pytest

from turing_sphere_b200 import _lib, gridForLmax, lmIndex, nlmCalc, validateConfig, ShtConfig

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(ts_\w+)\s*\(", src, flags=re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_bindings_cover_header():
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_layout_helpers_match_reference_rules():
    assert nlmCalc(255, 255) == 32896
    assert nlmCalc(63, 63) == 2080
    assert lmIndex(31, 31, 31) == nlmCalc(31, 31) - 1
    assert gridForLmax(63, 3) == (128, 256)
    assert gridForLmax(31, 1) == (32, 64)
    with pytest.raises(ValueError, match="nphi must be"):
        validateConfig(ShtConfig(31, 31, 32, 62))
    with pytest.raises(ValueError, match="mmax must be"):
        validateConfig(ShtConfig(31, 32, 32, 64))


def test_null_handles_are_rejected():
    L = _lib.lib()
    assert L.ts_ctx_destroy(None) == _lib.TS_ERR_INVALID
    assert L.ts_sht_plan_destroy(None) == _lib.TS_ERR_INVALID
    assert L.ts_sht_synth_dev(None, None, None, 1, None) == _lib.TS_ERR_INVALID
