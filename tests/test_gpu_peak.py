"""The FP64 FMA microbenchmark behind the FP64 roofline of the benchmark line."""
import pytest

import bench
import hawassi_c_b200 as hw

pytestmark = pytest.mark.gpu


def test_fp64_peak_is_plausible():
    v = hw.fp64_peak_tflops(0)
    print(f"FP64 FMA peak {v:.2f} TFLOP/s")
    assert 5.0 < v < 200.0


def test_fp64_roofline_entry():
    r = bench.fp64_roofline(2e12, 1000.0, 0, "k", "basis")
    assert r["bound"] == "fp64" and abs(r["achieved"] - 2.0) < 1e-12
    assert 0 < r["frac"] < 1 and r["peak"] > 5.0
