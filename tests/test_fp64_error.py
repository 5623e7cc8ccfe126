"""The fixed-point filter and the single-precision row solve against exact arithmetic
(oracle.fp64_error), on crops of the workloads: every int16 filtered value is within
4 Q14 LSB of the float64 four-pass filter, the mean error is below 0.6 LSB, and at
least 99.9% of pixels pick the same winning disparity; the float row solve gives the
double-precision solve's answer at 99.99% of pixels or more (beliefs within 1e-5),
and the whole int16/float path gives the double filter + double solve's answer within
0.5 px at 99.9% of pixels or more."""
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


@pytest.mark.parametrize("case", ["c1", "c2", "c3"])
def test_solve_error_statement(oracle, case):
    """The single-precision row solve against the same solve in double precision, on
    the same candidates and end to end (double filter + double solve)."""
    from doubleeye_b200 import synth
    if case == "c1":
        cfg, p = O.default_cfg(dmax=64, iters=10, census_hw=4), synth.fronto_planes(320, 200)
    elif case == "c2":
        cfg, p = O.default_cfg(dmax=96, iters=8), synth.slanted_planes(320, 200, 95)
    else:
        cfg, p = O.default_cfg(dmax=128, iters=12), synth.large_scene(400, 260, 127)
    s = fp64_error.solve_statement(oracle, cfg, p.left, p.right)
    assert s["solve_agreement"] >= 0.9999
    assert s["solve_max_disp_diff_px"] < 1e-4
    assert s["solve_max_belief_err"] < 1e-5
    assert s["e2e_agreement_0p5px"] >= 0.999
    assert abs(s["filled_f32"] - s["filled_f64"]) < 0.001
