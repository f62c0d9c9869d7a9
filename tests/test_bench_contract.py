"""bench.py's host-side contract on the CPU: argument defaults (graph replay
of the residual on for the single-system workloads, off for the c5 batch of
short solves) and the clock-record summary that decides whether a timed run
is kept (hw/thermal slowdowns are reported, power capping is kept)."""
import sys

import bench


def _args(argv):
    old = sys.argv
    sys.argv = ["bench.py"] + argv
    try:
        return bench.args()
    finally:
        sys.argv = old


def test_graph_replay_defaults():
    assert _args([]).use_graph == 1
    assert _args(["--workload", "c3"]).use_graph == 1
    assert _args(["--workload", "c5"]).use_graph == 0
    assert _args(["--use-graph", "0"]).use_graph == 0
    assert _args(["--workload", "c5", "--use-graph", "1"]).use_graph == 1
    a = _args([])
    assert (a.steps, a.warmup, a.gpus, a.impl) == (8, 3, 1, "ours")
    assert a.warmup >= 3


def _row(sm, power, hw="Not Active", thermal="Not Active", swt="Not Active", cap="Not Active"):
    # index, clocks.sm, clocks.max.sm, power.draw, active mask, hw_slowdown,
    # hw_thermal_slowdown, sw_thermal_slowdown, sw_power_cap
    return ["0", str(sm), "1965", str(power), "0x0", hw, thermal, swt, cap]


def test_clock_summary_reasons_and_loaded_median():
    c = bench.Clocks(0)
    c.rows = [_row(1965, 600.0), _row(1965, 620.0, cap="Active"), _row(345, 90.0)]
    s = c.summary()
    # the median is taken over samples under load (power above 250 W)
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 3
    c.rows = [_row(1500, 700.0, thermal="Active"), _row(1400, 700.0, hw="Active")]
    assert bench.Clocks.summary(c)["reasons"] == ["hw_slowdown", "hw_thermal_slowdown"]
    c.rows = []
    assert c.summary()["sm_mhz"] is None


def test_max_over_ranks_single_process():
    assert bench.max_over_ranks(0.25, 1) == 0.25
