"""The tcgen05 split-TF32 tensor-core Legendre path, through the C ABI, against
the f64 oracle.  Tolerance: relative L2 per transform <= 1e-5."""
import numpy as np
import pytest

from oracle import oracle as O
from turing_sphere_b200 import ShtConfig, ShtPlan

from .test_sht_gpu import scaled_spectrum

pytestmark = pytest.mark.gpu

TOL = 1e-5


def tc_plan(device, lmax, nlat, nphi, mmax=None):
    mmax = lmax if mmax is None else mmax
    return ShtPlan.create(device, ShtConfig(lmax, mmax, nlat, nphi), {"precision": "tf32x3"})


@pytest.mark.parametrize("lmax,nlat,nphi,mmax,batch", [
    (15, 16, 32, 15, 1),          # smallest tiles (N = 16)
    (31, 32, 64, 31, 1),          # the reference transformChecks grid
    (63, 96, 192, 63, 3),
    (127, 192, 384, 127, 70),     # two 64-field blocks, the second partial
    (255, 384, 768, 255, 2),      # one 192-latitude tile
    (255, 384, 768, 255, 16),     # the SHT configuration's batch sizes 16 and 256
    (255, 384, 768, 255, 256),
    (31, 33, 64, 31, 2),          # odd nlat: the equator row
    (40, 48, 96, 20, 5),          # mmax < lmax
])
def test_tc_parity_with_oracle(device, lmax, nlat, nphi, mmax, batch):
    plan = tc_plan(device, lmax, nlat, nphi, mmax)
    assert plan.precision == "tf32x3" and plan.tableBytes > 0
    ref = O.ShtReference(lmax, mmax, nlat, nphi)
    qs = np.stack([scaled_spectrum(lmax, mmax, 20 + b) for b in range(batch)])
    sp = plan.synth(qs, batch=batch).reshape(batch, -1)
    plan.status()
    for b in sorted({0, batch - 1}):
        s_cpu = ref.synth(qs[b].astype(np.float64))
        e_s = O.rel_l2(sp[b], s_cpu)
        s32 = s_cpu.astype(np.float32)
        e_a = O.rel_l2(plan.analys(s32), ref.analys(s32.astype(np.float64)))
        assert e_s < TOL and e_a < TOL, (b, e_s, e_a)
    back = plan.analys(sp, batch=batch).reshape(batch, -1)
    plan.status()
    assert O.rel_l2(back, qs) < TOL


def test_tc_latitude_tiles_lmax511(device):
    """nh = 384 latitudes: two 192-latitude tiles in the synthesis."""
    lmax, nlat, nphi = 511, 768, 1536
    plan = tc_plan(device, lmax, nlat, nphi)
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    q = scaled_spectrum(lmax, lmax, 9)
    s_cpu = ref.synth(q.astype(np.float64))
    assert O.rel_l2(plan.synth(q), s_cpu) < TOL
    s32 = s_cpu.astype(np.float32)
    assert O.rel_l2(plan.analys(s32), ref.analys(s32.astype(np.float64))) < TOL
    plan.status()


@pytest.mark.parametrize("lmax,nlat,nphi", [(127, 192, 384), (255, 384, 768)])
def test_tc_and_plain_both_within_tolerance(device, lmax, nlat, nphi):
    """Both precisions against f64 on the same input; they agree with each
    other to the sum of their errors."""
    a = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi))
    b = tc_plan(device, lmax, nlat, nphi)
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    q = scaled_spectrum(lmax, lmax, 4)
    s64 = ref.synth(q.astype(np.float64))
    sa, sb = a.synth(q), b.synth(q)
    ea, eb = O.rel_l2(sa, s64), O.rel_l2(sb, s64)
    print(f"synth relL2 vs f64: fp32 {ea:.2e}, tf32x3 {eb:.2e}")
    assert ea < TOL and eb < TOL
    assert O.rel_l2(sb, sa) < ea + eb + 1e-7
    s32 = s64.astype(np.float32)
    q64 = ref.analys(s32.astype(np.float64))
    fa, fb = O.rel_l2(a.analys(s32), q64), O.rel_l2(b.analys(s32), q64)
    print(f"analys relL2 vs f64: fp32 {fa:.2e}, tf32x3 {fb:.2e}")
    assert fa < TOL and fb < TOL


def test_w_stages_equal_analys_dev(device):
    """fourAnalysW then legAnalysW run exactly the kernels of analys_dev on a
    tensor-core plan, so the coefficients agree bit for bit; both stages are
    refused on an FP32 plan."""
    import torch
    lmax, nlat, nphi, B = 63, 96, 192, 70
    plan = tc_plan(device, lmax, nlat, nphi)
    rng = np.random.default_rng(5)
    spat = torch.from_numpy(rng.standard_normal((B, nlat * nphi)).astype(np.float32)).cuda()
    q1 = torch.empty(B, 2 * plan.nlm, device="cuda")
    q2 = torch.empty_like(q1)
    img = torch.zeros(plan.wimageBytes(B) // 4 + 1, device="cuda")
    plan.analys_dev(spat.data_ptr(), q1.data_ptr(), B)
    plan.stage_dev("fourAnalysW", spat.data_ptr(), img.data_ptr(), B)
    plan.stage_dev("legAnalysW", img.data_ptr(), q2.data_ptr(), B)
    torch.cuda.synchronize()
    plan.status()
    assert torch.equal(q1, q2)
    plain = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi), {"precision": "fp32"})
    assert plain.wimageBytes(B) == 0
    from turing_sphere_b200._lib import TsError
    with pytest.raises(TsError):
        plain.stage_dev("fourAnalysW", spat.data_ptr(), img.data_ptr(), B)


def test_autotuned_plan_keeps_parity(device):
    """TS_PLAN_AUTOTUNE times the tensor-core tiles and the FFT rows per CTA,
    keeps the fastest (reported in `shapes`) and stays within 1e-5; a second
    plan of the same grid reuses the choice."""
    lmax, nlat, nphi = 127, 192, 384
    cfg = ShtConfig(lmax, lmax, nlat, nphi)
    plan = ShtPlan.create(device, cfg, {"precision": "tf32x3", "autotune": True})
    sh = plan.shapes
    assert sh["tuned"] and sh["tc_lat_tile"] in (64, 96) and sh["tc_deg_tile"] in (64, 128)
    assert (sh["fft_p"], sh["fft_q"]) == (16, 12) and sh["fft_rows"] in (8, 16)
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    q = scaled_spectrum(lmax, lmax, 31)
    s_cpu = ref.synth(q.astype(np.float64))
    assert O.rel_l2(plan.synth(q), s_cpu) < TOL
    s32 = s_cpu.astype(np.float32)
    assert O.rel_l2(plan.analys(s32), ref.analys(s32.astype(np.float64))) < TOL
    plan.status()
    again = ShtPlan.create(device, cfg, {"precision": "tf32x3", "autotune": True})
    assert again.shapes == sh
    default = tc_plan(device, lmax, nlat, nphi)
    assert not default.shapes["tuned"] and default.shapes["tc_lat_tile"] == 96


def test_bounded_waits_time_out_and_the_plan_recovers(device):
    """Failure detection without a GPU fault: with the copy warp stalled (the
    plan's test hook) every bounded mbarrier wait of the tensor-core kernels
    runs out after a short limit; the kernels free their tensor memory and
    return, status() reports TS_ERR_TIMEOUT once, and with the stall lifted
    the same plan and context transform correctly again."""
    import time
    from turing_sphere_b200._lib import TS_ERR_TIMEOUT, TsError
    lmax, nlat, nphi = 31, 32, 64
    plan = tc_plan(device, lmax, nlat, nphi)
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    q = scaled_spectrum(lmax, lmax, 7)
    plan.testStall(True, wait_limit=4096)
    t0 = time.perf_counter()
    plan.synth(q)
    plan.analys(ref.synth(q.astype(np.float64)).astype(np.float32))
    assert time.perf_counter() - t0 < 30.0
    with pytest.raises(TsError) as ei:
        plan.status()
    assert ei.value.status == TS_ERR_TIMEOUT
    plan.status()  # reported once
    plan.testStall(False)
    s_cpu = ref.synth(q.astype(np.float64))
    assert O.rel_l2(plan.synth(q), s_cpu) < TOL
    s32 = s_cpu.astype(np.float32)
    assert O.rel_l2(plan.analys(s32), ref.analys(s32.astype(np.float64))) < TOL
    plan.status()
    fp32 = ShtPlan.create(device, ShtConfig(lmax, lmax, nlat, nphi), {"precision": "fp32"})
    with pytest.raises(TsError):
        fp32.testStall(True)


@pytest.mark.parametrize("lmax,nlat,nphi", [(255, 384, 768), (511, 768, 1536)])
def test_polar_skip_drops_work_not_accuracy(device, lmax, nlat, nphi):
    """The polar skip leaves out synthesis tiles and analysis latitude chunks
    whose table values are all below 1e-10 of their m's (tile's) largest; the
    high-m coefficients, the only ones it touches, stay within tolerance of
    the f64 oracle in both directions."""
    plan = tc_plan(device, lmax, nlat, nphi)
    assert plan.shapes["tc_skip_tiles"] > 0 and plan.shapes["tc_skip_chunks"] > 0
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    q = scaled_spectrum(lmax, lmax, 31)
    high = np.zeros_like(q)
    m0 = lmax // 2
    start = 2 * (m0 * (lmax + 1) - m0 * (m0 - 1) // 2)  # first coefficient of m = m0
    high[start:] = q[start:]
    s64 = ref.synth(high.astype(np.float64))
    assert O.rel_l2(plan.synth(high), s64) < TOL
    s32 = s64.astype(np.float32)
    q64 = ref.analys(s32.astype(np.float64))
    qa = plan.analys(s32)
    assert O.rel_l2(qa[start:], q64[start:]) < TOL
    plan.status()


def test_tc_lmax1023_parity(device):
    """The largest grid of the SHT configuration (lmax 1023 on 1536 x 3072):
    one field each way against the f64 oracle, with the polar skip active."""
    lmax, nlat, nphi = 1023, 1536, 3072
    plan = tc_plan(device, lmax, nlat, nphi)
    assert plan.shapes["tc_skip_chunks"] > 0
    ref = O.ShtReference(lmax, lmax, nlat, nphi)
    q = scaled_spectrum(lmax, lmax, 5)
    s64 = ref.synth(q.astype(np.float64))
    assert O.rel_l2(plan.synth(q), s64) < TOL
    s32 = s64.astype(np.float32)
    assert O.rel_l2(plan.analys(s32), ref.analys(s32.astype(np.float64))) < TOL
    plan.status()
