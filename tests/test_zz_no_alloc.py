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
