"""ORACLE — test infrastructure only.

ctypes wrapper over ``liboracle_sht.so`` (the f64 C restatement of the
reference's CPU transform, seeding and model steps; see oracle_sht.c) and over
``_ref/libshtb_spec.so`` (the reference's own bench/shtns/spec.h, compiled from
its sources).  Only tests, the smoke check and the benchmark's CPU-baseline leg
import this module; the product library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle_sht.so")
_REF = os.path.join(HERE, "_ref", "libshtb_spec.so")

_d = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_ip = C.POINTER(C.c_int)

MODELS = {"schnakenberg": 0, "brusselator": 1, "allencahn": 2, "linear": 3, "logistic": 4}


def build() -> None:
    """Compile the C restatement (and the reference shim when the tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    subprocess.run(["make", "-s", "-C", HERE, "ref"], check=True)


def _load():
    if not os.path.exists(_LIB):
        build()
    lib = C.CDLL(_LIB)
    lib.ors_nlm.restype = C.c_long
    lib.ors_nlm.argtypes = [C.c_int, C.c_int]
    lib.ors_lm_index.restype = C.c_long
    lib.ors_lm_index.argtypes = [C.c_int, C.c_int, C.c_int]
    lib.ors_validate.restype = C.c_int
    lib.ors_validate.argtypes = [C.c_int] * 4
    lib.ors_grid_for_lmax.argtypes = [C.c_int, C.c_int, _ip, _ip]
    lib.ors_gauss.argtypes = [C.c_int, _d, _d]
    lib.ors_legendre_coeffs.argtypes = [C.c_int, C.c_int, _d, _d]
    lib.ors_plan_create.restype = C.c_void_p
    lib.ors_plan_create.argtypes = [C.c_int] * 4
    lib.ors_plan_destroy.argtypes = [C.c_void_p]
    lib.ors_plan_nodes.argtypes = [C.c_void_p, _d, _d]
    for fn in ("ors_legendre_synth", "ors_fourier_synth", "ors_synth", "ors_fourier_analys",
               "ors_legendre_analys", "ors_analys"):
        getattr(lib, fn).argtypes = [C.c_void_p, _d, _d, C.c_int]
    lib.ors_random_spectrum.argtypes = [C.c_int, C.c_int, C.c_uint32, _f]
    lib.ors_seeded_spectrum.argtypes = [C.c_int, C.c_int, C.c_uint32, _f]
    lib.ors_seeded_noise.argtypes = [C.c_long, C.c_double, C.c_uint32, _f]
    lib.ors_eigenvalues.argtypes = [C.c_int, C.c_int, _d]
    lib.ors_model_species.restype = C.c_int
    lib.ors_model_species.argtypes = [C.c_int]
    lib.ors_model_step.restype = C.c_int
    lib.ors_model_step.argtypes = [C.c_void_p, C.c_int, _d, _d, C.c_int, C.c_int]
    lib.ors_synth_adjoint.argtypes = [C.c_void_p, _d, _d, C.c_int]
    lib.ors_analys_adjoint.argtypes = [C.c_void_p, _d, _d, C.c_int]
    lib.ors_model_adjoint.restype = C.c_int
    lib.ors_model_adjoint.argtypes = [C.c_void_p, C.c_int, _d, _d, C.c_int, C.c_int, _d, _d, _d,
                                      C.c_int]
    return lib


_lib = _load()


def nlm_calc(lmax: int, mmax: int) -> int:
    return int(_lib.ors_nlm(lmax, mmax))


def lm_index(lmax: int, l: int, m: int) -> int:
    return int(_lib.ors_lm_index(lmax, l, m))


def validate(lmax: int, mmax: int, nlat: int, nphi: int) -> int:
    return int(_lib.ors_validate(lmax, mmax, nlat, nphi))


def grid_for_lmax(lmax: int, pdeg: int) -> tuple[int, int]:
    a, b = C.c_int(), C.c_int()
    _lib.ors_grid_for_lmax(lmax, pdeg, C.byref(a), C.byref(b))
    return a.value, b.value


def gauss(n: int) -> tuple[np.ndarray, np.ndarray]:
    x = np.zeros(n)
    w = np.zeros(n)
    _lib.ors_gauss(n, x, w)
    return x, w


def legendre_coeffs(lmax: int, mmax: int) -> tuple[np.ndarray, np.ndarray]:
    amm = np.zeros(mmax + 1)
    ab = np.zeros(2 * nlm_calc(lmax, mmax))
    _lib.ors_legendre_coeffs(lmax, mmax, amm, ab)
    return amm, ab


def random_spectrum(lmax: int, mmax: int, seed: int) -> np.ndarray:
    q = np.zeros(2 * nlm_calc(lmax, mmax), dtype=np.float32)
    _lib.ors_random_spectrum(lmax, mmax, seed, q)
    return q


def seeded_spectrum(lmax: int, mmax: int, seed: int) -> np.ndarray:
    q = np.zeros(2 * nlm_calc(lmax, mmax), dtype=np.float32)
    _lib.ors_seeded_spectrum(lmax, mmax, seed, q)
    return q


def seeded_noise(npts: int, amp: float, seed: int) -> np.ndarray:
    out = np.zeros(npts, dtype=np.float32)
    _lib.ors_seeded_noise(npts, amp, seed, out)
    return out


def eigenvalues(lmax: int, mmax: int) -> np.ndarray:
    lam = np.zeros(2 * nlm_calc(lmax, mmax))
    _lib.ors_eigenvalues(lmax, mmax, lam)
    return lam


class ShtReference:
    """f64 direct-summation transform (reference.ts:13-119).

    ``threads`` = OpenMP threads (0 = all host cores, 1 = the single-threaded
    form the TypeScript runs)."""

    def __init__(self, lmax: int, mmax: int, nlat: int, nphi: int, threads: int = 0):
        self.lmax, self.mmax, self.nlat, self.nphi = lmax, mmax, nlat, nphi
        self.nlm = nlm_calc(lmax, mmax)
        self.threads = threads
        self._p = _lib.ors_plan_create(lmax, mmax, nlat, nphi)
        if not self._p:
            raise ValueError(f"invalid config lmax={lmax} mmax={mmax} nlat={nlat} nphi={nphi}")
        self.ct = np.zeros(nlat)
        self.wg = np.zeros(nlat)
        _lib.ors_plan_nodes(self._p, self.ct, self.wg)

    def __del__(self):
        p = getattr(self, "_p", None)
        if p:
            _lib.ors_plan_destroy(p)
            self._p = None

    def _run(self, fn, x, out_len):
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros(out_len)
        getattr(_lib, fn)(self._p, x, out, self.threads)
        return out

    def legendre_synth(self, qlm):
        return self._run("ors_legendre_synth", qlm, 2 * (self.mmax + 1) * self.nlat)

    def fourier_synth(self, fm):
        return self._run("ors_fourier_synth", fm, self.nlat * self.nphi)

    def synth(self, qlm):
        return self._run("ors_synth", qlm, self.nlat * self.nphi)

    def fourier_analys(self, spat):
        return self._run("ors_fourier_analys", spat, 2 * (self.mmax + 1) * self.nlat)

    def legendre_analys(self, gm):
        return self._run("ors_legendre_analys", gm, 2 * self.nlm)

    def analys(self, spat):
        return self._run("ors_analys", spat, 2 * self.nlm)

    def synth_adjoint(self, gbar):
        """S^T gbar, the transpose of synth with coefficients read as 2*nlm
        reals (m = 0 imaginary parts zero)."""
        return self._run("ors_synth_adjoint", gbar, 2 * self.nlm)

    def analys_adjoint(self, qbar):
        """A^T qbar, the transpose of analys (spectral cotangent -> grid)."""
        return self._run("ors_analys_adjoint", qbar, self.nlat * self.nphi)

    def model_step(self, model: str, params, state, nsteps: int):
        """Advance ``state`` (species x 2*nlm, f64) by ``nsteps`` IMEX steps."""
        mid = MODELS[model]
        S = int(_lib.ors_model_species(mid))
        st = np.ascontiguousarray(np.array(state, dtype=np.float64).reshape(S, 2 * self.nlm))
        prm = np.ascontiguousarray(np.array(params, dtype=np.float64))
        rc = _lib.ors_model_step(self._p, mid, prm, st, nsteps, self.threads)
        if rc != 0:
            raise ValueError(f"unknown model {model}")
        return st

    def model_adjoint(self, model: str, params, state, nsteps: int, every: int, final_bar):
        """Reverse mode of ``nsteps`` model steps from ``state`` (species x
        2*nlm) with checkpoints every ``every`` steps: returns
        (dL/d state, dL/d params) for dL/d(final state) = ``final_bar``."""
        mid = MODELS[model]
        S = int(_lib.ors_model_species(mid))
        st = np.ascontiguousarray(np.array(state, dtype=np.float64).reshape(S, 2 * self.nlm))
        fb = np.ascontiguousarray(np.array(final_bar, dtype=np.float64).reshape(S, 2 * self.nlm))
        prm = np.ascontiguousarray(np.array(params, dtype=np.float64))
        ib = np.zeros_like(st)
        pb = np.zeros(prm.size)
        rc = _lib.ors_model_adjoint(self._p, mid, prm, st, nsteps, every, fb, ib, pb,
                                    self.threads)
        if rc != 0:
            raise ValueError(f"unknown model {model}")
        return ib, pb


def rel_l2(a, b) -> float:
    """Relative L2 difference (digest.ts:55-63)."""
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    return float(np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b * b), 1e-300)))


class SpecRef:
    """The reference's own spec.h, compiled into _ref/libshtb_spec.so."""

    def __init__(self):
        if not os.path.exists(_REF):
            raise FileNotFoundError(_REF)
        lib = C.CDLL(_REF)
        lib.shtb_ref_grid_for_lmax.argtypes = [C.c_int, C.c_int, _ip, _ip]
        lib.shtb_ref_nlm.restype = C.c_long
        lib.shtb_ref_nlm.argtypes = [C.c_int, C.c_int]
        lib.shtb_ref_seeded_noise.argtypes = [C.c_long, C.c_double, C.c_uint, _f]
        lib.shtb_ref_seeded_spectrum.argtypes = [C.c_int, C.c_int, C.c_uint, _f]
        lib.shtb_ref_react_f32.argtypes = [C.c_int, _f, C.c_void_p, C.c_long, _f, C.c_void_p]
        lib.shtb_ref_react_f64.argtypes = [C.c_int, _d, C.c_void_p, C.c_long, _d, C.c_void_p]
        lib.shtb_ref_imex_f32.restype = C.c_float
        lib.shtb_ref_imex_f32.argtypes = [C.c_int, C.c_int, C.c_float, C.c_float, C.c_float]
        dp = C.POINTER(C.c_double)
        lib.shtb_ref_default_params.argtypes = [C.c_int, dp, dp, dp, dp, dp, dp]
        self.lib = lib

    @staticmethod
    def available() -> bool:
        return os.path.exists(_REF)

    def grid_for_lmax(self, lmax, pdeg):
        a, b = C.c_int(), C.c_int()
        self.lib.shtb_ref_grid_for_lmax(lmax, pdeg, C.byref(a), C.byref(b))
        return a.value, b.value

    def seeded_noise(self, npts, amp, seed):
        out = np.zeros(npts, dtype=np.float32)
        self.lib.shtb_ref_seeded_noise(npts, amp, seed, out)
        return out

    def seeded_spectrum(self, lmax, mmax, seed):
        q = np.zeros(2 * int(self.lib.shtb_ref_nlm(lmax, mmax)), dtype=np.float32)
        self.lib.shtb_ref_seeded_spectrum(lmax, mmax, seed, q)
        return q

    def react(self, model: int, u, v=None, f64=False):
        dt = np.float64 if f64 else np.float32
        u = np.ascontiguousarray(u, dtype=dt)
        n = u.size
        r1 = np.zeros(n, dtype=dt)
        r2 = np.zeros(n, dtype=dt) if v is not None else None
        vv = np.ascontiguousarray(v, dtype=dt) if v is not None else None
        fn = self.lib.shtb_ref_react_f64 if f64 else self.lib.shtb_ref_react_f32
        fn(model, u, vv.ctypes.data if vv is not None else None, n, r1,
           r2.ctypes.data if r2 is not None else None)
        return r1, r2

    def imex_f32(self, model, k, U, R, lam):
        return float(self.lib.shtb_ref_imex_f32(model, k, U, R, lam))

    def default_params(self, model):
        vals = [C.c_double() for _ in range(6)]
        self.lib.shtb_ref_default_params(model, *[C.byref(v) for v in vals])
        return {k: v.value for k, v in zip(("a", "b", "D1", "D2", "dt", "eps2"), vals)}
