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


CONTEXT_CHECK = r"""
import ctypes as C, sys
sys.path.insert(0, sys.argv[1])
from cuda.bindings import driver as cu
from turing_sphere_b200 import _lib
L = _lib.lib()
def current():
    err, ctx = cu.cuCtxGetCurrent()
    assert err == cu.CUresult.CUDA_SUCCESS, err
    return int(ctx)
cu.cuInit(0)
assert current() == 0  # this thread has never made a context current
h, p = C.c_void_p(), C.c_void_p()
assert L.ts_ctx_create(0, C.byref(h)) == 0
assert current() == 0, "ts_ctx_create left a context current"
assert L.ts_sht_plan_create(h, 15, 15, 16, 32, 0, C.byref(p)) == 0
assert current() == 0, "ts_sht_plan_create left a context current"
assert L.ts_sht_plan_destroy(p) == 0 and L.ts_ctx_destroy(h) == 0
assert current() == 0
print("ok")
"""


@pytest.mark.gpu
def test_calls_leave_the_callers_context_as_they_found_it(tmp_path):
    """Every C-ABI call makes its device current and gives the thread back the
    context it had: a thread that never touched CUDA has no current context
    after creating a context and a plan through the library (checked through
    the driver API in a fresh process)."""
    import subprocess
    import sys
    from tests.conftest import HAS_GPU
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    script = tmp_path / "ctx_check.py"
    script.write_text(CONTEXT_CHECK)
    r = subprocess.run([sys.executable, str(script), ROOT], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
