"""The roofline bench.py reports for a pair stage: the binding floor picks the
bound, and the fraction is achieved over peak in that bound's units."""
import bench


def test_hbm_bound_legendre_stage():
    # lmax 255, B 256: 268 MB moved, 6.47 GFLOP; 0.1 ms
    r = bench.stage_roofline("legAnalysW", 0.1, 268e6, 6.47e9, 3, 6650.0, 1590.0, "of fallback")
    assert r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert abs(r["achieved"] - 2680.0) < 1e-6 and abs(r["frac"] - 2680.0 / 6650.0) < 1e-12
    assert r["hbm_floor_us"] > r["tensor_floor_us"] and "of fallback" in r["peak_source"]


def test_tensor_bound_when_the_flops_dominate():
    r = bench.stage_roofline("legSynth", 1.0, 1e6, 1e12, 3, 6650.0, 1590.0, "of measured")
    assert r["bound"] == "tensor" and r["unit"] == "TFLOP/s"
    assert abs(r["frac"] - (1e12 / 1e-3 / 1e12) / 795.0) < 1e-12


def test_fourier_stage_is_hbm():
    r = bench.stage_roofline("fourSynth", 0.128, 503e6, 6.47e9, 3, 6650.0, 1590.0, "of fallback")
    assert r["bound"] == "hbm" and "tensor_floor_us" not in r
