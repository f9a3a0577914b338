"""Host logic of bench.py (no GPU): workload members, the per-workload DRAM
traffic of the roofline (the capture of the same launch shape, else the
nearest capture scaled by algorithmic bytes per launch), and the arguments."""
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402


def test_members_of_plain_and_mixed_workloads():
    assert bench.members("gst_1500x100") == [("gst_1500x100", None)]
    assert bench.members("gst_coreg3_600x40") == [("gst_coreg3_600x40", None)]
    mixed = bench.members("mixed_8x1200_16x600")
    assert mixed == [("gst_coreg2_600x40", 8), ("gst_600x40", 16)]
    assert bench.config_of("gst_600x40")["nb"] == 1


def test_traffic_of_the_captured_launch_shape_is_taken_as_is():
    t, src = bench.roofline_traffic("gst_1500x100", "panel", (1500, 6, 6))
    assert t == 2590.0e6 and "same launch shape" in src


def test_traffic_of_another_shape_is_scaled_by_algorithmic_bytes():
    t, src = bench.roofline_traffic("gst_4000x250", "panel", (4000, 6, 2))
    scale = bench.panel_bytes_per_launch(4000, 6, 2) / bench.panel_bytes_per_launch(1500, 6, 6)
    assert abs(t - 2590.0e6 * scale) < 1.0
    assert "scaled" in src
    t2, _ = bench.roofline_traffic("x", "gemm", (1500, 6, 24))
    assert abs(t2 - 346851328.0 * 4.0) < 1.0  # four times the matrices per launch
    t3, src3 = bench.roofline_traffic("x", "gemm", (1500, 6, 12))
    assert t3 == 706.0e6 and "same launch shape" in src3


def test_default_arguments():
    a = bench.parse([])
    assert (a.workload, a.batch, a.precision, a.factor_precision, a.fd_steps) == \
        ("gst_1500x100", 6, "i8slice", "auto", 3)


def test_auto_factor_precision_by_block_size():
    """"auto" takes the 8-bit-slice Schur updates only when every model of the
    group has blocks of at least AUTO_I8_FACTOR_MIN_BLOCK; an FP64 selected
    inversion (the fallback included) always factors in FP64."""
    from types import SimpleNamespace as NS

    from dalia_b200.model import AUTO_I8_FACTOR_MIN_BLOCK as B, _factor_arith

    big, small = NS(b=B), NS(b=B - 1)
    assert _factor_arith("auto", [big], "i8slice") == "i8slice"
    assert _factor_arith("auto", [big, small], "i8slice") == "fp64"
    assert _factor_arith("auto", [big], "fp64") == "fp64"
    assert _factor_arith("i8slice", [small], "i8slice") == "i8slice"
    assert _factor_arith("i8slice", [big], "fp64") == "fp64"
    assert _factor_arith("fp64", [big], "i8slice") == "fp64"
