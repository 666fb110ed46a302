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


def test_served_stream_admission_by_estimate():
    """The c5 stream keeps exactly the queries whose estimated count and scan
    work fit the budget (an impossible pattern always fits, a budget of zero
    scanned entries admits nothing that scans)."""
    import tdfs_b200 as T
    g = T.gen_er(4096, 16.0, 0).set_labels(4, 2)
    none = "v 0 9\nv 1 9\nv 2 9\ne 0 1 1\ne 0 2 1\ne 1 2 1\n"   # label 9 occurs nowhere: 0 matches, 0 scans
    tri = "v 0 1\nv 1 1\nv 2 1\ne 0 1 1\ne 0 2 1\ne 1 2 1\n"
    wide = "v 0 1\nv 1 1\nv 2 1\nv 3 1\ne 0 1 1\ne 1 2 1\ne 1 3 1\n"  # a labeled star: many matches
    texts = [none, tri, wide]
    assert bench.admit_stream(T, g, texts, 1e12, 1e12) == [0, 1, 2]
    assert bench.admit_stream(T, g, texts, 1e12, 0) == [0]
    est_wide = T.estimate(g, T.PatternPreprocessor(text=wide, labeled=True), 1024, 2).matches
    assert est_wide > 0
    assert 2 not in bench.admit_stream(T, g, texts, est_wide / 1000, 1e12)
