"""The fixed-point filter against exact arithmetic (oracle.fp64_error): on crops of
the workloads, every int16 filtered value is within 4 Q14 LSB of the float64
four-pass filter, the mean error is below 0.6 LSB, and at least 99.9% of pixels pick
the same winning disparity.  At full size the same statement reads 2.4-3.1 LSB max,
0.40-0.42 mean and 99.988-99.998% agreement (C1-C4)."""
import pytest

from oracle import fp64_error
from oracle import oracle as O


@pytest.mark.parametrize("case", ["c1", "c2", "c3"])
def test_filter_error_statement(oracle, case):
    from doubleeye_b200 import synth
    if case == "c1":
        cfg, p = O.default_cfg(dmax=64, census_hw=4), synth.fronto_planes(320, 200)
    elif case == "c2":
        cfg, p = O.default_cfg(dmax=96), synth.slanted_planes(320, 200, 95)
    else:
        cfg, p = O.default_cfg(dmax=128), synth.large_scene(400, 260, 127)
    s = fp64_error.statement(oracle, cfg, p.left, p.right)
    assert s["values"] > 1_000_000
    assert s["max_err_lsb"] <= 4.0
    assert s["mean_err_lsb"] < 0.6
    assert s["winner_agreement"] >= 0.999
