"""The benchmark's algorithmic-byte accounting (bench.py), on the CPU: which
spectral products ran fused with their x transform, the words each kernel
category moves, and the once-a-step FD divergence check."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402

NPTS = 256 * 256 * 128


def test_fused_mode_from_profile_categories():
    assert bench.fused_mode({"fft_x_r2c": {}, "spec_products": {}}) == ""
    assert bench.fused_mode({"spec_products_fx": {}, "spec_products": {}, "fft_x_r2c": {}}) == "mom"
    assert bench.fused_mode({"spec_products_fx": {}}) == "all"


def _words(kernel, fused):
    return bench.alg_bytes_step(kernel, NPTS, 4, "sp", fused=fused) / (3 * NPTS * 4)


def test_spectral_words_per_category():
    # separate kernels: products 18 + temperature 7, x forward of 8 + 3 fields
    assert _words("spec_products", "") == 25
    assert _words("fft_x_r2c", "") == 22
    # momentum fused: 18 words; the temperature products and their x transform stay
    assert _words("spec_products_fx", "mom") == 18
    assert _words("spec_products", "mom") == 7
    assert _words("fft_x_r2c", "mom") == 6
    # both fused: 18 + 7, nothing left in the separate categories
    assert _words("spec_products_fx", "all") == 25
    assert _words("spec_products", "all") == 0
    assert _words("fft_x_r2c", "all") == 0


def test_fusion_removes_exactly_the_physical_products_round_trip():
    cats = ("spec_products", "fft_x_r2c", "spec_products_fx")
    sep = sum(_words(c, "") for c in cats)
    mom = sum(_words(c, "mom") for c in cats)
    both = sum(_words(c, "all") for c in cats)
    # each fused physical product field is no longer written and read back
    assert sep - mom == 8 * 2
    assert sep - both == (8 + 3) * 2


def test_fd_divergence_check_counted_once_a_step():
    n = 512 * 384 * 256
    assert bench.alg_bytes_step("div_check", n, 4, "fd") == 3 * n * 4
    assert bench.alg_bytes_step("rhs_momentum", n, 4, "fd") == 13 * 3 * n * 4


def test_statistics_bytes_per_point():
    # FP64: u, v, w, t plus uhx, vhy snapshots (FD) and 11 accumulators read and written
    assert bench.stats_bytes_per_point("fd", 8) == 6 * 8 + 11 * 2 * 8
    # FP32 window sums, folded into the FP64 sums once a window
    w = bench.STATS_WINDOW
    assert abs(bench.stats_bytes_per_point("sp", 4) - (4 * 4 + 11 * 2 * 4 + 11 * (4 + 16 + 4) / w)) < 1e-12
    # without a temperature equation: 8 accumulators and no T
    assert bench.stats_bytes_per_point("fd", 8, with_t=False) == 5 * 8 + 8 * 2 * 8
