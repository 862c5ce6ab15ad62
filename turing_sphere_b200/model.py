"""A .m model compiled and running on a B200 (src/mgpu/model.ts, plan.ts,
session.ts of the reference), over the C ABI.

GpuModel.create compiles `init` and `step` for the plan's grid (NVRTC, sm_100a)
with ``batch`` independent instances; ModelSession picks the grid for a
registry model and seeds it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .layout import ShtConfig, gridForLmax
from .noise import seededNoise
from .sht import Device, ShtPlan


class ModelCompileError(Exception):
    """A rejected model source, located in the file (errors.ts:14-31)."""

    def __init__(self, message, start=None, end=None, fn=None):
        super().__init__(message)
        self.start, self.end, self.fn = start, end, fn


def formatFailure(e: Exception, source: str) -> str:
    """errors.ts:93-105: message with 1-based line/column and function."""
    if not isinstance(e, ModelCompileError):
        return str(e)
    where = []
    if e.start is not None and 0 <= e.start <= len(source):
        before = source[:e.start]
        where.append(f"line {before.count(chr(10)) + 1}, column {e.start - before.rfind(chr(10))}")
    if e.fn:
        where.append(f"in {e.fn}()")
    return f"{e} ({', '.join(where)})" if where else str(e)


def _raise_compile(err, rc, dev):
    msg = err.message.decode() or (_lib.lib().ts_last_error(dev).decode())
    if rc == _lib.TS_ERR_COMPILE:
        raise ModelCompileError(msg, err.start if err.start >= 0 else None,
                                err.end if err.end >= 0 else None, err.fn.decode() or None)
    raise _lib.TsError(rc, msg)


def eigenvalues(cfg: ShtConfig) -> np.ndarray:
    """model.ts:46-56: l(l+1) per coefficient, duplicated over re/im."""
    out = []
    for m in range(cfg.mmax + 1):
        for l in range(m, cfg.lmax + 1):
            out += [l * (l + 1)] * 2
    return np.asarray(out, dtype=np.float32)


class GpuModel:
    def __init__(self, device, sht, handle, paramNames, state, view, batch):
        self.device, self.sht, self.handle = device, sht, handle
        self.paramNames, self.state, self.view, self.batch = paramNames, state, view, batch
        self.npts = sht.cfg.nlat * sht.cfg.nphi
        self.nlm = sht.nlm
        self._sizes = {s: 2 * self.nlm for s in state}
        self._sizes.update({"lam": 2 * self.nlm, "noise": self.npts})
        for v in view:
            self._sizes.setdefault(v, self.npts)

    @staticmethod
    def create(device: Device, sht: ShtPlan, source: str, paramNames, state, view,
               batch: int = 1) -> "GpuModel":
        """GpuModel.create (model.ts:103-163)."""
        h = C.c_void_p()
        err = _lib.CompileError()
        rc = _lib.lib().ts_model_compile(
            sht.handle, source.encode(), _lib.cstr_array(state), len(state),
            _lib.cstr_array(view), len(view), _lib.cstr_array(paramNames), len(paramNames),
            batch, C.byref(h), C.byref(err))
        if rc != _lib.TS_OK:
            _raise_compile(err, rc, device.handle)
        return GpuModel(device, sht, h, list(paramNames), list(state), list(view), batch)

    def _check(self, rc):
        _lib.check(rc, self.device.handle)

    def setParams(self, params) -> None:
        """plan.ts:410-420: by name; missing or non-finite -> 0.  A list of
        dicts (one per instance) sets a parameter sweep."""
        if isinstance(params, (list, tuple)):
            vals = np.array([[float(p.get(k, 0.0)) for k in self.paramNames] for p in params],
                            dtype=np.float32)
            self._check(_lib.lib().ts_model_set_params_batched(
                self.handle, _lib.fptr(np.ascontiguousarray(vals)), len(params), len(self.paramNames)))
            return
        vals = np.array([float(params.get(k, 0.0)) for k in self.paramNames], dtype=np.float32)
        self._check(_lib.lib().ts_model_set_params(self.handle, _lib.fptr(vals), vals.size))

    def upload(self, name: str, data) -> None:
        d = np.ascontiguousarray(data, dtype=np.float32).ravel()
        rc = _lib.lib().ts_model_upload(self.handle, name.encode(), _lib.fptr(d), d.size)
        if rc in (_lib.TS_ERR_NOT_FOUND, _lib.TS_ERR_SIZE):
            raise ValueError(_lib.lib().ts_last_error(self.device.handle).decode())
        self._check(rc)

    def init(self, noise=None) -> None:
        if noise is None:
            self._check(_lib.lib().ts_model_init(self.handle, None, 0))
            return
        d = np.ascontiguousarray(noise, dtype=np.float32).ravel()
        rc = _lib.lib().ts_model_init(self.handle, _lib.fptr(d), d.size)
        if rc == _lib.TS_ERR_SIZE:
            raise ValueError(_lib.lib().ts_last_error(self.device.handle).decode())
        self._check(rc)

    def step(self, steps: int = 1) -> None:
        self._check(_lib.lib().ts_model_step(self.handle, steps))

    def forwardBackward(self, nsteps: int, every: int, finalBar):
        """The adjoint's forward/backward pair (no reference counterpart; the
        autograd.Function of this path): advance ``nsteps`` steps keeping a
        state checkpoint every ``every`` steps, then run the hand-written
        adjoint backwards.  ``finalBar``: dL/d(final state), a dict state ->
        (instances, 2 nlm) array (missing states: zero).  Returns
        (dL/d(initial state) as such a dict, dL/d(params) as an
        (instances, nparams) float64 array in ``paramNames`` order)."""
        ns, B, n2 = len(self.state), self.batch, 2 * self.nlm
        fb = np.zeros((ns, B, n2), dtype=np.float32)
        for i, s in enumerate(self.state):
            if s in finalBar:
                fb[i] = np.asarray(finalBar[s], dtype=np.float32).reshape(B, n2)
        ib = np.zeros_like(fb)
        pb = np.zeros((B, max(len(self.paramNames), 1)), dtype=np.float64)
        self._check(_lib.lib().ts_model_forward_backward(
            self.handle, nsteps, every, _lib.fptr(fb), _lib.fptr(ib), _lib.dptr(pb)))
        return {s: ib[i] for i, s in enumerate(self.state)}, pb[:, :len(self.paramNames)]

    def lossGradient(self, nsteps: int, every: int, finalBarOf):
        """Gradient of a loss of the final state: ``finalBarOf(final)`` maps
        the final states (dict state -> (instances, 2 nlm) array) to
        dL/d(final state); the model ends at the final state, as after
        ``step(nsteps)``.  Returns what forwardBackward returns."""
        self.snapshotState()
        self.step(nsteps)
        final = {s: self.read(s).reshape(self.batch, -1) for s in self.state}
        self.restoreState()
        return self.forwardBackward(nsteps, every, finalBarOf(final))

    def setGraphs(self, enable: bool) -> None:
        """Run steps as captured CUDA graphs (default) or launch them eagerly."""
        self._check(_lib.lib().ts_model_set_graphs(self.handle, 1 if enable else 0))

    def snapshotState(self) -> None:
        self._check(_lib.lib().ts_model_snapshot(self.handle))

    def restoreState(self) -> None:
        self._check(_lib.lib().ts_model_restore(self.handle))

    def read(self, name: str, instance: int | None = None) -> np.ndarray:
        """All instances ([batch, n]) or one; instance 0 alone is a plain read."""
        n = self._sizes.get(name)
        if n is None:
            n = self._lookup_size(name)
        out = np.empty(n * self.batch, dtype=np.float32)
        rc = _lib.lib().ts_model_read(self.handle, name.encode(), _lib.fptr(out), out.size)
        if rc == _lib.TS_ERR_NOT_FOUND:
            raise KeyError(_lib.lib().ts_last_error(self.device.handle).decode())
        self._check(rc)
        out = out.reshape(self.batch, n)
        if instance is not None:
            return out[instance]
        return out[0] if self.batch == 1 else out

    def _lookup_size(self, name):
        ptr, cnt = C.c_void_p(), C.c_long()
        rc = _lib.lib().ts_model_value_ptr(self.handle, name.encode(), C.byref(ptr), C.byref(cnt))
        if rc != _lib.TS_OK:
            raise KeyError(_lib.lib().ts_last_error(self.device.handle).decode())
        return cnt.value

    def valueBuffer(self, name: str) -> tuple[int, int]:
        ptr, cnt = C.c_void_p(), C.c_long()
        self._check(_lib.lib().ts_model_value_ptr(self.handle, name.encode(), C.byref(ptr),
                                                  C.byref(cnt)))
        return ptr.value, cnt.value

    def describe(self) -> dict:
        out = {}
        for which, key in ((0, "init"), (1, "step")):
            buf = C.create_string_buffer(1 << 16)
            self._check(_lib.lib().ts_model_describe(self.handle, which, buf, len(buf)))
            out[key] = [l for l in buf.value.decode().splitlines() if l]
        return out

    def counts(self, which: str = "step") -> tuple[int, int]:
        k, n = C.c_int(), C.c_int()
        self._check(_lib.lib().ts_model_counts(self.handle, 0 if which == "init" else 1,
                                               C.byref(k), C.byref(n)))
        return k.value, n.value

    def generatedSource(self) -> str:
        buf = C.create_string_buffer(1 << 20)
        self._check(_lib.lib().ts_model_source(self.handle, buf, len(buf)))
        return buf.value.decode()

    def destroy(self) -> None:
        if self.handle:
            _lib.lib().ts_model_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


class ModelSession:
    """One running model (session.ts:28-218): grid by gridForLmax, mmax = lmax."""

    def __init__(self, device, model, cfg, sht, displaySht, gpu, params, oversample):
        self.device, self.model, self.cfg, self.sht = device, model, cfg, sht
        self.gpu, self._params, self._displaySht = gpu, params, displaySht
        self._oversample = oversample
        self.npts = cfg.nlat * cfg.nphi
        self.t = 0.0
        self.steps = 0

    @staticmethod
    def create(device, model, params, lmax, source=None, oversample=1, batch=1, grid=None,
               precision="fp32") -> "ModelSession":
        oversample = max(1, int(round(oversample)))
        nlat, nphi = grid if grid is not None else gridForLmax(lmax, model.pdeg)
        cfg = ShtConfig(lmax, lmax, nlat, nphi)
        sht = ShtPlan.create(device, cfg, {"precision": precision})
        display = None
        if oversample > 1:
            display = ShtPlan.create(device, ShtConfig(lmax, lmax, oversample * nlat,
                                                       oversample * nphi))
        gpu = GpuModel.create(device, sht, source or model.source, [p.key for p in model.params],
                              model.state, model.species, batch)
        gpu.setParams(params)
        return ModelSession(device, model, cfg, sht, display, gpu, params, oversample)

    @property
    def oversample(self) -> int:
        return self._oversample

    @property
    def viewSht(self) -> ShtPlan:
        return self._displaySht or self.sht

    def setOversample(self, oversample: int) -> None:
        os_ = max(1, int(round(oversample)))
        if os_ == self._oversample:
            return
        old = self._displaySht
        self._displaySht = None if os_ == 1 else ShtPlan.create(
            self.device, ShtConfig(self.cfg.lmax, self.cfg.mmax, os_ * self.cfg.nlat,
                                   os_ * self.cfg.nphi))
        self._oversample = os_
        if old:
            old.destroy()

    def seed(self, seed: int) -> None:
        """Run `init` from seeded noise (instance k uses seed + k)."""
        noise = np.concatenate([seededNoise(self.npts, self.model.seedAmp, seed + k)
                                for k in range(self.gpu.batch)])
        self.gpu.init(noise)
        self.t = 0.0
        self.steps = 0

    def setParams(self, params) -> None:
        self._params = params
        self.gpu.setParams(params)

    def step(self, n: int = 1) -> None:
        self.gpu.step(n)
        dt = self._params[0].get("dt", 0) if isinstance(self._params, list) else self._params.get("dt", 0)
        self.t += n * dt
        self.steps += n

    def sync(self) -> None:
        self.device.sync()

    def measure(self, n: int) -> float:
        """ms/step of n steps, leaving state, t and steps untouched (session.ts:179-187)."""
        import time
        self.gpu.snapshotState()
        self.device.sync()
        t0 = time.perf_counter()
        self.gpu.step(n)
        self.device.sync()
        ms = (time.perf_counter() - t0) * 1e3 / n
        self.gpu.restoreState()
        self.device.sync()
        return ms

    def read(self, name: str, instance=None) -> np.ndarray:
        return self.gpu.read(name, instance)

    def readSpecies(self, k: int) -> np.ndarray:
        """Species k at render resolution: the model's field, or the state
        synthesised on the oversampled grid (session.ts:201-207)."""
        if not self._displaySht:
            return self.read(self.model.species[k])
        # the spectral state (2 nlm floats) comes back to the host and the
        # display plan synthesises it through its own staging buffers
        q = self.gpu.read(self.model.state[k], 0)
        return self._displaySht.synth(q)

    def describe(self) -> dict:
        return self.gpu.describe()

    def destroy(self) -> None:
        self.gpu.destroy()
        if self._displaySht:
            self._displaySht.destroy()
        self.sht.destroy()


class ModelGroup:
    """Ragged batches: several GpuModels (e.g. instances at different lmax,
    each on its own plan) stepped together, every step one CUDA graph whose
    branches run the models concurrently (ts_model_group_*)."""

    def __init__(self, models):
        self.models = list(models)
        arr = (C.c_void_p * len(self.models))(*[m.handle.value if hasattr(m.handle, "value")
                                                 else m.handle for m in self.models])
        h = C.c_void_p()
        dev = self.models[0].device
        _lib.check(_lib.lib().ts_model_group_create(arr, len(self.models), C.byref(h)), dev.handle)
        self.handle, self.device = h, dev

    def step(self, n: int = 1) -> None:
        _lib.check(_lib.lib().ts_model_group_step(self.handle, n), self.device.handle)

    def destroy(self) -> None:
        if self.handle:
            _lib.lib().ts_model_group_destroy(self.handle)
            self.handle = None
