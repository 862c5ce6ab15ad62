"""The allocation-free synthesis entry point, through the C ABI.

ts_sht_synth_noalloc is for callers that cannot let the library call
cudaMalloc (hosts that own all device memory, or loops that must not stall on
cudaMalloc's implicit device synchronisation).  Its result must equal
ts_sht_synth_dev's on the same input, call after call, although every call
reuses one fixed scratch array.  This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from turing_sphere_b200 import ShtConfig, ShtPlan, _lib

pytestmark = pytest.mark.gpu

TOL = 1e-6


def test_noalloc_synth_matches_allocating_synth(device):
    import torch
    L = _lib.lib()
    lmax, nlat, nphi = 127, 192, 384
    plan = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi))
    B = 8
    rng = np.random.default_rng(5)
    for call in range(2):
        q = torch.from_numpy(rng.standard_normal((B, 2 * plan.nlm)).astype(np.float32)).cuda()
        want = torch.empty(B, nlat * nphi, device="cuda")
        got = torch.full((B, nlat * nphi), float("nan"), device="cuda")
        torch.cuda.synchronize()
        _lib.check(L.ts_sht_synth_dev(plan.handle, q.data_ptr(), want.data_ptr(), B, None),
                   device.handle)
        _lib.check(L.ts_sht_synth_noalloc(plan.handle, q.data_ptr(), got.data_ptr(), B, None),
                   device.handle)
        device.sync()
        w, g = want.cpu().numpy(), got.cpu().numpy()
        assert np.isfinite(g).all()
        assert O.rel_l2(g, w) <= TOL, (call, O.rel_l2(g, w))


def test_noalloc_rejects_batches_beyond_the_scratch_limit(device):
    import torch
    L = _lib.lib()
    lmax, nlat, nphi = 255, 384, 768
    plan = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi))
    B = 64  # 64 * 256 * 384 * 8 bytes = 48 MiB > 16 MiB
    q = torch.zeros(B, 2 * plan.nlm, device="cuda")
    s = torch.zeros(B, nlat * nphi, device="cuda")
    rc = L.ts_sht_synth_noalloc(plan.handle, q.data_ptr(), s.data_ptr(), B, None)
    assert rc == _lib.TS_ERR_SIZE
    assert b"fixed" in L.ts_last_error(device.handle)


def _synth_both(L, plan, q, B, device):
    import torch
    nq = plan.cfg.nlat * plan.cfg.nphi
    want = torch.empty(B, nq, device="cuda")
    got = torch.full((B, nq), float("nan"), device="cuda")
    torch.cuda.synchronize()
    _lib.check(L.ts_sht_synth_dev(plan.handle, q.data_ptr(), want.data_ptr(), B, None),
               device.handle)
    _lib.check(L.ts_sht_synth_noalloc(plan.handle, q.data_ptr(), got.data_ptr(), B, None),
               device.handle)
    device.sync()
    return want.cpu().numpy(), got.cpu().numpy()


def test_noalloc_fills_the_scratch_array_exactly_at_its_limit(device, parity):
    """The largest batch the 16 MiB array holds at lmax 255 (21 fields: the
    count the size error reports) gives the allocating synthesis's result in
    every field, the last one included, twice in a row; one field more is
    refused with TS_ERR_SIZE."""
    import torch
    L = _lib.lib()
    lmax, nlat, nphi = 255, 384, 768
    plan = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi))
    per_field = (lmax + 1) * nlat * 8
    B = (16 << 20) // per_field
    assert B == 21
    rng = np.random.default_rng(11)
    for call in range(2):
        q = torch.from_numpy(rng.standard_normal((B, 2 * plan.nlm)).astype(np.float32)).cuda()
        want, got = _synth_both(L, plan, q, B, device)
        assert np.isfinite(got).all()
        for f in (0, B - 1):
            parity(f"noalloc lmax255 B=21 call{call} field{f} vs synth_dev",
                   O.rel_l2(got[f], want[f]), TOL)
    q = torch.zeros(B + 1, 2 * plan.nlm, device="cuda")
    s = torch.zeros(B + 1, nlat * nphi, device="cuda")
    assert L.ts_sht_synth_noalloc(plan.handle, q.data_ptr(), s.data_ptr(), B + 1,
                                  None) == _lib.TS_ERR_SIZE
    assert b"at most 21 fields" in L.ts_last_error(device.handle)
    plan.destroy()


def test_noalloc_on_a_tensor_core_plan_matches_the_f64_oracle(device, parity):
    """On a tensor-core plan the allocation-free call runs the FP32 Legendre
    recurrence (the tensor-core path needs an operand image the plan grows on
    demand); its result still meets the 1e-5 transform bar against the f64
    oracle, on two calls in a row.  Inputs: Gaussian coefficients scaled by
    (l+1)^-1, the transform workload's spectrum."""
    import torch
    L = _lib.lib()
    lmax, nlat, nphi = 127, 192, 384
    plan = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi), {"precision": "tf32x3"})
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    B = 4
    l_of = np.concatenate([np.arange(m, lmax + 1) for m in range(lmax + 1)])
    for call in range(2):
        rng = np.random.default_rng(7 + call)
        qh = rng.standard_normal((B, plan.nlm, 2)) / (l_of[None, :, None] + 1.0)
        qh[:, :lmax + 1, 1] = 0.0  # m = 0 imaginary parts
        qh = np.ascontiguousarray(qh.reshape(B, -1), dtype=np.float32)
        q = torch.from_numpy(qh).cuda()
        want, got = _synth_both(L, plan, q, B, device)
        for f in (0, B - 1):
            parity(f"noalloc tf32x3 plan lmax127 call{call} field{f}",
                   O.rel_l2(got[f], ref.synth(qh[f].astype(np.float64))), 1e-5)
        assert O.rel_l2(got, want) <= 1e-5
    plan.destroy()
