"""Host-side pieces of bench.py: the step edge ranges, the committed ncu
record it reads into the roofline, the reference arm's engine-free inputs, and
the clock record without nvidia-smi."""
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


def test_profile_record_holds_only_for_its_kernel_sources(tmp_path):
    """An ncu record enters the roofline only when it was captured on the
    kernel sources built here (their digest is stored with it)."""
    path = tmp_path / "ncu.json"
    rec = {"dram_bytes_per_launch": 1.0e6, "issue_active_pct": 30.0, "command": "ncu ..."}
    path.write_text(json.dumps({"c13": dict(rec, kernel_sources=bench.kernel_source_digest()),
                                "c2": dict(rec, kernel_sources="0" * 16)}))
    assert bench.measured_profile("c13", str(path))["issue_active_pct"] == 30.0
    assert bench.measured_profile("c2", str(path)) is None
    assert bench.measured_profile("c4", str(path)) is None
    committed = os.path.join(bench.ROOT, "profiles", "match_kernel_ncu.json")
    if os.path.exists(committed):
        for wl, r in json.load(open(committed)).items():
            assert "ncu" in r["command"] and "--clock-control none" in r["command"], wl


def test_reference_arm_inputs_without_the_engine(tmp_path):
    """The reference arm writes its graph and patterns with the host-only
    tdfs_convert tool: the same files the engine's generators give, and the
    process that does it never loads libtdfs_b200.so."""
    import subprocess
    import sys
    import tdfs_b200 as T
    code = ("import sys, bench; E = bench.graph_via_convert('er_l', sys.argv[1]); "
            "print(E); [print(repr(bench.convert_pattern(*s))) for s in bench.c3_pattern_specs()]; "
            "import os; maps = open('/proc/self/maps').read(); print('libtdfs_b200' in maps, 'tdfs_b200' in sys.modules)")
    out = subprocess.run([sys.executable, "-c", code, str(tmp_path / "g")], cwd=bench.ROOT, capture_output=True,
                         text=True, check=True).stdout.splitlines()
    g = T.gen_er(4096, 16.0, 0).set_labels(4, 2)
    assert int(out[0]) == g.nedges
    r = T.read_csr(str(tmp_path / "g"), labeled=True)
    assert (r.colidx == g.colidx).all() and (r.labels == g.labels).all()
    import ast
    assert [ast.literal_eval(l) for l in out[1:9]] == [T.gen_pattern(*s) for s in bench.c3_pattern_specs()]
    assert out[9] == "False False"


def test_workloads_name_the_configs():
    desc, key, pats, slices = bench.workload("c13")
    assert key == "er_l" and slices == 1 and len(pats) == 12
    assert [lab for _, _, lab in pats] == [False] * 4 + [True] * 8
    assert bench.workload("c2")[3] == 1000 and bench.workload("c4")[3] == 500000


def test_clock_record_without_nvidia_smi():
    c = bench.ClockSampler(0)  # never started
    rec = c.stop()
    assert rec["sm_mhz"] is None and rec["reasons"] == ["nvidia-smi unavailable"]


def test_served_stream_queries():
    """The config-5 stream: seeded, 3-7 vertices, labels in [0, 4), every
    query a valid connected pattern in matching order."""
    import tdfs_b200 as T
    a = bench.c5_queries(T.gen_pattern, 300)
    assert a == bench.c5_queries(T.gen_pattern, 300)
    ks = [T.PatternPreprocessor(text=t, labeled=True).nnodes for t in a]
    assert min(ks) == 3 and max(ks) == 7
