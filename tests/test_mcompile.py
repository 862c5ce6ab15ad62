"""The .m compiler front end and code generation, without a GPU
(ts_model_check: parse, specialise, schedule, NVRTC compile for sm_100a)."""
import ctypes as C

import pytest

from turing_sphere_b200 import _lib, mModels, defaultParams
from turing_sphere_b200.model import formatFailure, ModelCompileError


def check(source, state=("U",), view=("u",), params=(), lmax=15, nlat=16, nphi=32, batch=1,
          precision=0):
    buf = C.create_string_buffer(1 << 16)
    k, n = C.c_int(), C.c_int()
    err = _lib.CompileError()
    rc = _lib.lib().ts_model_check(lmax, lmax, nlat, nphi, source.encode(),
                                   _lib.cstr_array(list(state)), len(state),
                                   _lib.cstr_array(list(view)), len(view),
                                   _lib.cstr_array(list(params)), len(params), batch, precision, buf,
                                   len(buf), C.byref(k), C.byref(n), C.byref(err))
    if rc != _lib.TS_OK:
        raise ModelCompileError(err.message.decode(), err.start, err.end, err.fn.decode())
    init, step = buf.value.decode().split("====\n")
    return k.value, n.value, init.splitlines(), step.splitlines()


EXPECTED_KERNELS = {"schnakenberg": 5, "brusselator": 5, "allencahn": 2}


@pytest.mark.parametrize("model", mModels, ids=lambda m: m.key)
def test_models_fuse_one_kernel_per_line(model):
    """test/modelChecks.ts:17-21: one element-wise statement per source line;
    here they further fuse into 3 launches per step."""
    k, n, init, step = check(model.source, model.state, model.species,
                             [p.key for p in model.params], lmax=31, nlat=48, nphi=96)
    assert k == EXPECTED_KERNELS[model.key]
    assert n == 3
    assert step[-3].startswith("legsyn") and step[-2].startswith("phase")
    assert "fused" in step[-1]
    assert sum(l.startswith("synth") for l in step) == len(model.state)
    assert sum(l.startswith("analys") for l in step) == len(model.state)


@pytest.mark.parametrize("grid", [(63, 96, 192), (255, 384, 768), (127, 192, 384)])
@pytest.mark.parametrize("precision", [0, 1], ids=["fp32", "tf32x3"])
def test_schnakenberg_compiles_on_large_grids(grid, precision):
    m = mModels[0]
    lmax, nlat, nphi = grid
    k, n, init, step = check(m.source, m.state, m.species, [p.key for p in m.params], lmax, nlat,
                             nphi, batch=64, precision=precision)
    # tensor-core plans with many instances run the IMEX update as its own
    # coalesced element-wise stage instead of the analysis epilogue, and their
    # Legendre synthesis is two kernels (operand relayout, tcgen05 contraction)
    assert n == (3 if precision == 0 else 5)
    if precision:
        assert step[-1].startswith("specew") or "spectral" in step[-1], step


LINEAR = open(__file__.replace("test_mcompile.py", "models/linear.m")).read()
LOGISTIC = open(__file__.replace("test_mcompile.py", "models/logistic.m")).read()


@pytest.mark.parametrize("which", ["schnakenberg", "brusselator", "allencahn", "linear",
                                   "logistic"])
def test_step_adjoint_generates_and_compiles(which):
    """TS_CHECK_ADJOINT: the reverse-mode kernels of every model's step
    (symbolic derivatives of its element-wise statements) compile for
    sm_100a; the IMEX update's parameter derivatives are emitted."""
    if which in ("linear", "logistic"):
        src = LINEAR if which == "linear" else LOGISTIC
        params = ["c", "D", "dt"] if which == "linear" else ["r", "D", "dt"]
        state, view = ("U",), ("u",)
    else:
        m = [x for x in mModels if x.key == which][0]
        src, params, state, view = m.source, [p.key for p in m.params], m.state, m.species
    buf = C.create_string_buffer(1 << 20)
    k, n = C.c_int(), C.c_int()
    err = _lib.CompileError()
    rc = _lib.lib().ts_model_check(31, 31, 48, 96, src.encode(), _lib.cstr_array(list(state)),
                                   len(state), _lib.cstr_array(list(view)), len(view),
                                   _lib.cstr_array(list(params)), len(params), 4,
                                   _lib.TS_CHECK_SOURCE | _lib.TS_CHECK_ADJOINT, buf, len(buf),
                                   C.byref(k), C.byref(n), C.byref(err))
    assert rc == _lib.TS_OK, err.message.decode()
    code = buf.value.decode()
    assert "ts_adj_r0" in code and "atomicAdd(io.pbar" in code


@pytest.mark.parametrize("src,msg", [
    ("function [U, u] = step(U, lam)\n u = synth(U);\n Un = U;\nend\n",
     "must define a function named 'init'"),
    (LINEAR.replace("(U, lam, c, D, dt)", "(U, lam, c, D, dt, zz)"),
     "takes an argument named 'zz', which this app does not provide"),
    (LINEAR.replace("analys(c * u)", "analys(c * u .* U)"), "implicit expansion"),
    (LINEAR.replace("analys(c * u)", "analys(u * u)"), "matrix '*' is not supported"),
    (LINEAR.replace("analys(c * u)", "analys(u .^ c)"), "literal integer exponent"),
    (LINEAR.replace("analys(c * u)", "analys(u .^ 2.5)"), "literal integer exponent"),
    (LINEAR.replace("  u = synth(U);\n  Un", "  u = synth(U);\n  if c\n  end\n  Un"),
     "'if' is not supported"),
    (LINEAR.replace("analys(c * u)", "analys(u(3))"), "indexing 'u' is not supported"),
    (LINEAR + "\nfunction y = helper(x)\n  y = x;\nend\n",
     None),  # an unused helper is fine
    (LINEAR.replace("analys(c * u)", "analys(helper(u))") +
     "\nfunction y = helper(x)\n  y = x;\nend\n", "is a function defined in this model"),
    (LINEAR.replace("analys(c * u)", "analys(c * w)"), "undefined function or variable 'w'"),
    (LINEAR.replace("analys(c * u)", "analys(c * u"), "expected"),
    (LINEAR.replace("analys(c * u)", "analys(U)"), "analys requires a 512x1 array, got 2x136"),
    (LINEAR.replace("Un = (U", "Vn = (U"), "declares the output 'Un' but never assigns it"),
    (LINEAR.replace("analys(c * u)", "analys(c * u + ones(3, 1))"), "only grid"),
])
def test_compile_errors(src, msg):
    params = ["c", "D", "dt"]
    if msg is None:
        check(src, params=params)
        return
    with pytest.raises(ModelCompileError, match=msg.replace("(", r"\(").replace(")", r"\)")
                       .replace("*", r"\*").replace(".", r"\.")):
        check(src, params=params)


def test_error_location_is_in_the_source():
    src = LINEAR.replace("analys(c * u)", "analys(c * u .* U)")
    with pytest.raises(ModelCompileError) as ei:
        check(src, params=["c", "D", "dt"])
    e = ei.value
    assert e.fn == "step"
    assert e.start is not None and src[e.start:e.end].startswith("c * u .* U")
    text = formatFailure(e, src)
    line = src[:e.start].count("\n") + 1
    assert f"line {line}" in text and "in step()" in text


def test_builtins_powers_and_scalars_compile():
    src = """
function [U, u] = init(noise)
  U = analys(noise);
  u = synth(U);
end
function [Un, u] = step(U, lam, c, D, dt)
  u = synth(U);
  k = 2 * c;            % derived scalar
  e = exp(1) + pi;      % exact scalar
  w = max(u, 0) - abs(u) .* tanh(u) + sqrt(abs(u)) + u.^-2 - -u.^4 + e;
  Un = (U + dt * analys(k * w)) ./ (1 + (dt * D) * lam);
end
"""
    k, n, init, step = check(src, params=["c", "D", "dt"])
    assert k == 3 and n == 3


def test_comments_and_continuations():
    src = LINEAR.replace("Un = (U + dt * analys(c * u))",
                         "%{\nblock comment\n%}\n  Un = (U + dt * ... continued\n analys(c * u))")
    check(src, params=["c", "D", "dt"])


def test_round_rounds_halfway_cases_to_even():
    """WGSL round (src/mgpu/wgsl.ts:64 maps .m round to it) takes a halfway
    value to the even integer; the generated CUDA calls rintf (round to
    nearest even), not roundf (halfway cases away from zero)."""
    src = LINEAR.replace("analys(c * u)", "analys(c * round(u))")
    buf = C.create_string_buffer(1 << 20)
    k, n = C.c_int(), C.c_int()
    err = _lib.CompileError()
    rc = _lib.lib().ts_model_check(15, 15, 16, 32, src.encode(), _lib.cstr_array(["U"]), 1,
                                   _lib.cstr_array(["u"]), 1, _lib.cstr_array(["c", "D", "dt"]),
                                   3, 1, _lib.TS_CHECK_SOURCE, buf, len(buf), C.byref(k),
                                   C.byref(n), C.byref(err))
    assert rc == _lib.TS_OK, err.message.decode()
    code = buf.value.decode()
    assert "rintf(" in code and "roundf(" not in code
