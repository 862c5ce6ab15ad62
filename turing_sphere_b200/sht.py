"""Spherical-harmonic transform plans on a B200 (src/sht/sht.ts of the reference).

``Device`` stands where the reference's GPUDevice does (requestShtDevice,
sht.ts:495-513); ``ShtPlan`` mirrors ShtPlan: ``create`` validates the config
and builds the tables, ``synth``/``analys`` are blocking host-array transforms
that raise on a length mismatch, and the ``*_dev`` forms take device pointers
(the encodeSynthInto/encodeAnalysInto counterpart) and only enqueue work.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from .layout import ShtConfig, nlmCalc, validateConfig


class Device:
    """One CUDA device and stream (ts_ctx)."""

    def __init__(self, ordinal: int = 0):
        h = C.c_void_p()
        rc = _lib.lib().ts_ctx_create(ordinal, C.byref(h))
        _lib.check(rc, None)
        self.handle = h
        self.ordinal = ordinal

    @property
    def name(self) -> str:
        buf = C.create_string_buffer(256)
        _lib.check(_lib.lib().ts_ctx_device_name(self.handle, buf, 256), self.handle)
        return buf.value.decode()

    def set_stream(self, stream_ptr: int | None) -> None:
        _lib.check(_lib.lib().ts_ctx_set_stream(self.handle, stream_ptr), self.handle)

    @property
    def stream(self) -> int:
        return _lib.lib().ts_ctx_stream(self.handle) or 0

    def sync(self) -> None:
        _lib.check(_lib.lib().ts_sync(self.handle), self.handle)

    def destroy(self) -> None:
        if self.handle:
            _lib.lib().ts_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


_default_device: Device | None = None


def requestShtDevice(ordinal: int = 0) -> Device:
    """The process-wide device for ``ordinal`` (requestShtDevice, sht.ts:495-513)."""
    global _default_device
    if _default_device is None or _default_device.ordinal != ordinal:
        _default_device = Device(ordinal)
    return _default_device


PRECISIONS = {"fp32": _lib.TS_PREC_FP32, "tf32x3": _lib.TS_PREC_TF32X3,
              "bf16x3": _lib.TS_PREC_BF16X3}
FOURIERS = {"auto": _lib.TS_FOURIER_AUTO, "fft": _lib.TS_FOURIER_FFT, "dft": _lib.TS_FOURIER_DFT}


class ShtPlan:
    """A transform plan for one (lmax, mmax, nlat, nphi) grid."""

    def __init__(self, device: Device, cfg: ShtConfig, handle, info):
        self.device = device
        self.cfg = cfg
        self.handle = handle
        self.nlm = nlmCalc(cfg.lmax, cfg.mmax)
        self.fourierMode = "dft" if info.fourier == _lib.TS_FOURIER_DFT else "fft"
        self.precision = {v: k for k, v in PRECISIONS.items()}[info.precision]
        self.fftRadices = [info.fft_radix[i] for i in range(info.fft_stages)]
        self.tableBytes = info.table_bytes
        # kernel shapes in use: tensor-core tiles, two-phase FFT split, FFT rows per CTA
        self.shapes = {"tc_lat_tile": info.tc_lat_tile, "tc_deg_tile": info.tc_deg_tile,
                       "fft_p": info.fft_p, "fft_q": info.fft_q, "fft_rows": info.fft_rows,
                       "tuned": bool(info.tuned), "tc_skip_tiles": info.tc_skip_tiles,
                       "tc_skip_chunks": info.tc_skip_chunks}
        x = np.zeros(cfg.nlat)
        w = np.zeros(cfg.nlat)
        _lib.check(_lib.lib().ts_sht_plan_nodes(handle, _lib.dptr(x), _lib.dptr(w)), device.handle)
        self.cosTheta = x
        self.gaussWeights = w
        self.theta = np.arccos(x)
        self.legLat = (cfg.nlat + 1) // 2

    @staticmethod
    def create(device: Device, cfg: ShtConfig, opts: dict | None = None) -> "ShtPlan":
        """ShtPlan.create (sht.ts:166-183).  opts: fourier = auto|fft|dft,
        precision = fp32|tf32x3|bf16x3, autotune = True to time the kernel
        shapes at creation (the choice is in `shapes`)."""
        opts = opts or {}
        validateConfig(cfg)
        flags = PRECISIONS[opts.get("precision", "fp32")] | FOURIERS[opts.get("fourier", "auto")]
        if opts.get("autotune"):
            flags |= _lib.TS_PLAN_AUTOTUNE
        h = C.c_void_p()
        rc = _lib.lib().ts_sht_plan_create(device.handle, cfg.lmax, cfg.mmax, cfg.nlat, cfg.nphi,
                                           flags, C.byref(h))
        if rc == _lib.TS_ERR_INVALID:
            raise ValueError(_lib.lib().ts_last_error(device.handle).decode())
        _lib.check(rc, device.handle)
        info = _lib.PlanInfo()
        _lib.check(_lib.lib().ts_sht_plan_info(h, C.byref(info)), device.handle)
        return ShtPlan(device, cfg, h, info)

    # ---- blocking host-array transforms (sht.ts:414-461)
    def synth(self, qlm, batch: int = 1) -> np.ndarray:
        q = np.ascontiguousarray(qlm, dtype=np.float32).ravel()
        npts = self.cfg.nlat * self.cfg.nphi
        if q.size != 2 * self.nlm * batch:
            raise ValueError(f"qlm must have length {2 * self.nlm * batch}")
        out = np.empty(npts * batch, dtype=np.float32)
        _lib.check(_lib.lib().ts_sht_synth(self.handle, _lib.fptr(q), q.size, _lib.fptr(out),
                                           out.size, batch), self.device.handle)
        return out

    def analys(self, spat, batch: int = 1) -> np.ndarray:
        s = np.ascontiguousarray(spat, dtype=np.float32).ravel()
        npts = self.cfg.nlat * self.cfg.nphi
        if s.size != npts * batch:
            raise ValueError(f"spat must have length {npts * batch}")
        out = np.empty(2 * self.nlm * batch, dtype=np.float32)
        _lib.check(_lib.lib().ts_sht_analys(self.handle, _lib.fptr(s), s.size, _lib.fptr(out),
                                            out.size, batch), self.device.handle)
        return out

    def roundtrip(self, qlm, batch: int = 1, out=None) -> np.ndarray:
        """analys(synth(qlm)) per field with host arrays in and out and the
        grid kept on the device: the round trip of scripts/bench-sht.ts:190-217
        as one blocking call (ts_sht_roundtrip, pipelined over chunks of
        fields).  `out` may be a preallocated float32 array (e.g. page-locked)."""
        q = np.ascontiguousarray(qlm, dtype=np.float32).ravel()
        if q.size != 2 * self.nlm * batch:
            raise ValueError(f"qlm_in must have length {2 * self.nlm * batch}")
        if out is None:
            out = np.empty(q.size, dtype=np.float32)
        self.roundtrip_ptr(q.ctypes.data, out.ctypes.data, batch)
        return out

    def roundtrip_ptr(self, in_ptr: int, out_ptr: int, batch: int = 1) -> None:
        """ts_sht_roundtrip on raw host pointers (2 nlm floats per field each)."""
        n = 2 * self.nlm * batch
        _lib.check(_lib.lib().ts_sht_roundtrip(self.handle, in_ptr, n, out_ptr, n, batch),
                   self.device.handle)

    # ---- device-pointer transforms (encodeSynthInto / encodeAnalysInto)
    def synth_dev(self, qlm_ptr: int, spat_ptr: int, batch: int = 1, stream: int | None = None):
        _lib.check(_lib.lib().ts_sht_synth_dev(self.handle, qlm_ptr, spat_ptr, batch, stream),
                   self.device.handle)

    def analys_dev(self, spat_ptr: int, qlm_ptr: int, batch: int = 1, stream: int | None = None):
        _lib.check(_lib.lib().ts_sht_analys_dev(self.handle, spat_ptr, qlm_ptr, batch, stream),
                   self.device.handle)

    def synth_adjoint_dev(self, gbar_ptr: int, qbar_ptr: int, batch: int = 1,
                          stream: int | None = None):
        """qbar = S^T gbar: the transpose of synth_dev (grid -> spectral)."""
        _lib.check(_lib.lib().ts_sht_synth_adjoint_dev(self.handle, gbar_ptr, qbar_ptr, batch,
                                                       stream), self.device.handle)

    def analys_adjoint_dev(self, qbar_ptr: int, gbar_ptr: int, batch: int = 1,
                           stream: int | None = None):
        """gbar = A^T qbar: the transpose of analys_dev (spectral -> grid)."""
        _lib.check(_lib.lib().ts_sht_analys_adjoint_dev(self.handle, qbar_ptr, gbar_ptr, batch,
                                                        stream), self.device.handle)

    def wimageBytes(self, batch: int) -> int:
        """Bytes of the tensor-core analysis operand image for `batch` fields
        (0 on an FP32 plan)."""
        return int(_lib.lib().ts_sht_wimage_bytes(self.handle, batch))

    def stage_dev(self, stage: str, src_ptr: int, dst_ptr: int, batch: int = 1,
                  stream: int | None = None):
        """One stage alone (encodeStage, sht.ts:362-401): legSynth | fourSynth |
        fourAnalys | legAnalys, and on tensor-core plans the two stages of
        analys_dev: fourAnalysW (grid -> operand image) | legAnalysW (image ->
        coefficients)."""
        fn = {"legSynth": "ts_sht_leg_synth_dev", "fourSynth": "ts_sht_fourier_synth_dev",
              "fourAnalys": "ts_sht_fourier_analys_dev", "legAnalys": "ts_sht_leg_analys_dev",
              "fourAnalysW": "ts_sht_fourier_analys_w_dev",
              "legAnalysW": "ts_sht_leg_analys_w_dev"}[stage]
        _lib.check(getattr(_lib.lib(), fn)(self.handle, src_ptr, dst_ptr, batch, stream),
                   self.device.handle)

    def testStall(self, stall: bool, wait_limit: int = 0) -> None:
        """Failure-detection test hook (tensor-core plans): make the kernels'
        bounded waits run out (stall) or restore normal operation."""
        _lib.check(_lib.lib().ts_sht_plan_test_stall(self.handle, 1 if stall else 0, wait_limit),
                   self.device.handle)

    def status(self) -> None:
        """Raise TsError(TS_ERR_TIMEOUT) if a tensor-core kernel gave up a wait."""
        _lib.check(_lib.lib().ts_sht_plan_status(self.handle), self.device.handle)

    def destroy(self) -> None:
        if self.handle:
            _lib.lib().ts_sht_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass


def flop_per_pair(lmax: int, mmax: int, nlat: int, nphi: int) -> float:
    """Algorithmic flops of one synth + one analys of one field:
    2 * (2 nlm nlat [parity-folded Legendre] + 2.5 nphi log2(nphi) nlat [FFT])."""
    nlm = (mmax + 1) * (lmax + 1) - mmax * (mmax + 1) // 2
    return 2.0 * (2.0 * nlm * nlat + 2.5 * nphi * math.log2(nphi) * nlat)


def bytes_per_pair(lmax: int, mmax: int, nlat: int, nphi: int) -> float:
    """Minimum HBM bytes of one synth + one analys: read+write of the
    coefficients (8 nlm) and of the grid (4 nlat nphi), both directions."""
    nlm = (mmax + 1) * (lmax + 1) - mmax * (mmax + 1) // 2
    return 2.0 * (8.0 * nlm + 4.0 * nlat * nphi)
