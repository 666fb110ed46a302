"""Host-side pieces of bench.py: the step edge ranges, the committed traffic
record it reads into the roofline, and the clock record without nvidia-smi."""
import json
import os

import bench


def test_step_ranges_whole_graph_and_slices():
    warm, timed = bench.step_ranges(1000, 1, 5, 3)
    assert warm == [(0, 1000)] * 3 and timed == [(0, 1000)] * 5
    E = 6_000_000
    warm, timed = bench.step_ranges(E, 1000, 5, 3)
    # timed slices j = (s + 1/2) * 1000 / 5: 100, 300, ..., 900, each 1/1000 of the edges
    assert timed == [(j * E // 1000, (j + 1) * E // 1000) for j in (100, 300, 500, 700, 900)]
    assert all(b < e for b, e in warm + timed)
    assert not set(warm) & set(timed)  # warm-up never touches a timed slice


def test_traffic_record_is_read_per_workload():
    with open(os.path.join(bench.ROOT, "profiles", "match_kernel_traffic.json")) as f:
        rec = json.load(f)
    for wl in ("c2", "c4"):
        assert bench.measured_traffic(wl) == rec[wl]["dram_bytes_per_launch"] > 0
        assert "ncu" in rec[wl]["command"] and "--clock-control none" in rec[wl]["command"]
    assert bench.measured_traffic("c1") is None


def test_clock_record_without_nvidia_smi():
    c = bench.ClockSampler(0)  # never started
    rec = c.stop()
    assert rec["sm_mhz"] is None and rec["reasons"] == ["nvidia-smi unavailable"]
