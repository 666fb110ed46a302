"""GPU counts through the C ABI vs the CPU oracle, bit-exact (uint64).

Graphs are the seeded synthetic inputs of the benchmark configs at sizes the
oracle finishes in seconds: the ER graph of the small configs at full size
(n=4096, average degree 16, seed 0; labels uniform in [0,4), seed 2),
reduced Chung-Lu power-law graphs (hubs far above the per-level buffer so
chunked production, stealing and the split queue all run), a reduced R-MAT
graph, and complete graphs with closed-form counts."""
import json
import math
import os
import random

import numpy as np
import pytest

from tests.golden.make_golden import random_pattern
from tests.patterns import CYCLE4, HOUSE, TRIANGLE, clique, reference_patterns

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

OPTION_SETS = [
    {},                                              # defaults (stealing + split queue on, merge window)
    {"steal": 0},                                    # plain persistent DFS
    {"merge_window": -1},                            # per-lane search only
    {"chunk_cap": 64, "warps_per_block": 4},         # tiny buffers: many refills
    {"merge_window": 256, "chunk_cap": 128, "blocks_per_sm": 1},
    {"fixed_stage": -1, "edge_chunk": 32, "steal_min": 8},  # no last-level staging
    {"edge_chunk": 1, "steal_first": 2, "split_after_us": -1},  # one edge per ticket, eager splits
    {"edge_chunk": 4, "blocks_per_sm": 2, "steal_first": 32},
    {"lane_list": 64, "chunk_cap": 128},   # longer lists in the flattened last-level pass
    {"lane_list": -1},                     # one warp-wide pass per last-level sibling
    {"split_rush_us": 10, "steal_first": 2},            # tail rush after 10 us
    {"split_rush_us": 1, "split_after_us": 400, "fixed_stage": -1},  # long gate, 1 us in the tail
    {"label_index": -1, "leaf_steal_min": -1},          # labeled level 0 over every edge id; leaves stealable
    {"level_hoist": -1, "fixed_stage": -1, "label_rows": -1},  # every level produced per node; whole rows
    {"chunk_cap": 64, "split_after_us": -1, "steal_first": 2},  # tiny buffers, eager splits of hoisted levels
    {"tail_count": -1, "lane_list": -1, "dead_prune": -1},  # every level enumerated, no dead-subtree checks
]


class Case:
    def __init__(self, T, po, csr, labeled):
        self.csr = csr
        self.dev = T.GraphPreprocessor(csr=csr, labeled=labeled)
        self.ora = po.Graph(csr.rowptr.copy(), csr.colidx.copy(),
                            None if csr.labels is None else csr.labels.copy())
        self.T, self.po = T, po
        self.want = {}

    def check(self, text, labeled, **opt):
        T, po = self.T, self.po
        key = (text, labeled)
        if key not in self.want:  # one oracle run per pattern, whatever the option sets
            self.want[key] = po.count(self.ora, po.Plan(text, labeled))
        want = self.want[key]
        got = T.count(self.dev, T.PatternPreprocessor(text=text, labeled=labeled), T.default_options(**opt))
        assert got.count == want, (text, labeled, opt, got.count, want)
        return want


@pytest.fixture(scope="module")
def er(T, po):
    return Case(T, po, T.gen_er(4096, 16.0, 0).set_labels(4, 2), True)


@pytest.fixture(scope="module")
def cl(T, po):
    # reduced Chung-Lu: 50k vertices, 150k edges, gamma 2.1, cap 3000 (max degree ~2.2k > buffers)
    return Case(T, po, T.gen_chung_lu(50000, 150000, 2.1, 3000, 1).set_labels(4, 2), True)


@pytest.fixture(scope="module")
def cl_small(T, po):
    return Case(T, po, T.gen_chung_lu(20000, 60000, 2.1, 600, 1).set_labels(4, 2), True)


def test_er_unlabeled_config_patterns(er):
    # the 4-clique count of this sparse ER graph is 0 (expected ~0.04)
    assert er.check(clique(4), False) == 0
    assert er.check(TRIANGLE, False) > 0 and er.check(CYCLE4, False) > 0
    for _, text in reference_patterns():
        er.check(text, False)


def test_er_labeled_reference_patterns(er):
    for _, text in reference_patterns():
        er.check(text, True)


def test_er_labeled_random_6_7(er):
    rng = random.Random(3)
    for t in range(16):
        er.check(random_pattern(6 + t % 2, 0.4, 4, rng), True)


@pytest.mark.parametrize("opt", OPTION_SETS)
def test_er_option_sets(er, opt):
    for text in [TRIANGLE, CYCLE4, clique(4), HOUSE]:
        er.check(text, False, **opt)
    rng = random.Random(5)
    for t in range(4):
        er.check(random_pattern(5 + t % 3, 0.5, 4, rng), True, **opt)


@pytest.mark.parametrize("opt", OPTION_SETS)
def test_powerlaw_unlabeled(cl, opt):
    for text in [TRIANGLE, CYCLE4, clique(4), clique(5)]:
        cl.check(text, False, **opt)


def test_powerlaw_house_and_reference(cl_small):
    for text in [HOUSE] + [t for _, t in reference_patterns()]:
        cl_small.check(text, False)
        cl_small.check(text, True)


def test_powerlaw_labeled_random(cl):
    rng = random.Random(3)
    for t in range(10):
        cl.check(random_pattern(4 + t % 4, 0.45, 4, rng), True)


@pytest.mark.parametrize("opt", [{}, {"chunk_cap": 64}, {"tail_count": -1}, {"dead_prune": -1},
                                 {"level_hoist": -1}])
def test_independent_tails(er, cl_small, T, opt):
    """Patterns whose last two or three vertices hang only on earlier ones and
    not on each other: a node at the root of that tail counts its leaves by
    inclusion-exclusion over their candidate sets, on labeled plans taken from
    hoisted levels' core sets and the last vertex's fixed set where those are
    anchored earlier (level_hoist=-1: every set built per node).  With 64-entry
    buffers the power-law graph's hub sets do not fit and those nodes descend
    the ordinary way; tail_count=-1 enumerates everywhere."""
    for i in range(8):  # the config-3 patterns: five of them have such a tail
        er.check(T.gen_pattern(6 + i % 2, 0.4, 4, 3000 + i), True, **opt)
    rng = random.Random(12)
    for t in range(6):
        cl_small.check(random_pattern(5 + t % 3, 0.35, 4, rng), True, **opt)
    # unlabeled tails (no order condition between the tail's vertices)
    rng = random.Random(11)
    for t in range(23):
        text = random_pattern(5 + t % 2, 0.5, 1, rng)
        if t in (6, 7, 14, 15, 20, 22):
            er.check(text, False, **opt)
    rng = random.Random(11)
    for t in range(16):
        text = random_pattern(5 + t % 3, 0.35, 1, rng)
        if t == 15:
            cl_small.check(text, False, **opt)


def test_rmat_reduced(T, po):
    case = Case(T, po, T.gen_rmat(14, 16, 0.57, 0.19, 0.19, 4), False)
    for text in [TRIANGLE, clique(4)]:
        case.check(text, False)


@pytest.mark.parametrize("n", [12, 40])
def test_complete_graph_closed_form(T, n):
    rowptr = np.arange(0, n * (n - 1) + 1, n - 1, dtype=np.int64)
    colidx = np.array([j for i in range(n) for j in range(n) if j != i], dtype=np.int32)
    G = T.GraphPreprocessor(rowptr=rowptr, colidx=colidx, labels=np.ones(n, np.int32), labeled=True)
    for k, text in [(3, TRIANGLE), (4, CYCLE4), (5, HOUSE), (5, clique(5)), (6, clique(6)), (7, clique(7))]:
        for labeled in (False, True):
            got = T.count(G, T.PatternPreprocessor(text=text, labeled=labeled)).count
            assert got == math.perm(n, k)


@pytest.mark.parametrize("chunk", [0, 1, 4])
def test_edge_shards_sum_to_total(er, T, chunk):
    """Level-0 chunks dealt round-robin over shards (the multi-GPU split), with
    the default 32-edge deal and with explicit finer chunks, over the whole
    graph and over a slice; batched launches deal the same way."""
    P = T.PatternPreprocessor(text=CYCLE4)
    total = T.count(er.dev, P).count
    parts = [T.count(er.dev, P, T.shard_options(r, 3, edge_chunk=chunk)).count for r in range(3)]
    assert sum(parts) == total and min(parts) > 0
    b, e = 1000, 7000
    part = T.count(er.dev, P, T.default_options(edge_begin=b, edge_end=e)).count
    shards = [T.count_batch(er.dev, [P], T.shard_options(r, 4, edge_begin=b, edge_end=e, edge_chunk=chunk))[0][0]
              for r in range(4)]
    assert sum(shards) == part


@pytest.mark.parametrize("chunk", [0, 1, 4])
def test_labeled_ranges_and_shards_through_the_label_index(er, cl, T, chunk):
    """Labeled level-0 tickets walk the label index; edge ranges and
    round-robin shards still cover exactly the same edge ids as without it."""
    rng = random.Random(23)
    for case in (er, cl):
        text = random_pattern(5, 0.5, 4, rng)
        P = T.PatternPreprocessor(text=text, labeled=True)
        total = T.count(case.dev, P).count
        assert total == T.count(case.dev, P, T.default_options(label_index=-1)).count
        E = case.csr.nedges
        b, e = E // 5, E // 2
        part = T.count(case.dev, P, T.default_options(edge_begin=b, edge_end=e)).count
        assert part == T.count(case.dev, P, T.default_options(edge_begin=b, edge_end=e, label_index=-1)).count
        assert part == case.po.count(case.ora, case.po.Plan(text, True), 0, b, e)
        shards = [T.count(case.dev, P, T.shard_options(r, 3, edge_begin=b, edge_end=e, edge_chunk=chunk)).count
                  for r in range(3)]
        assert sum(shards) == part


def test_cli_matches_reference_line_format(T, tmp_path):
    import subprocess
    g = T.gen_er(4096, 16.0, 0).set_labels(4, 2)
    prefix = str(tmp_path / "snap.txt")
    g.write(prefix)
    pat = tmp_path / "tri.g"
    pat.write_text(TRIANGLE)
    for exe, labeled in (("ulb", False), ("lb", True)):
        out = subprocess.run([os.path.join(T.BIN_DIR, exe), prefix, str(pat)], capture_output=True, text=True,
                             check=True).stdout.strip().splitlines()[-1]
        path, ms, cnt = out.split("\t")
        assert path == str(pat) and float(ms) > 0
        G = T.GraphPreprocessor(prefix, labeled=labeled)
        assert int(cnt) == T.count(G, T.PatternPreprocessor(str(pat), labeled)).count


def test_reference_build_counts(T):
    """Counts printed by the reference's own CUDA build (tests/golden/ref_counts.json),
    except its recorded failures (ref_known_failures.json), where the oracle's
    count is expected."""
    path = os.path.join(GOLDEN, "ref_counts.json")
    if not os.path.exists(path):
        pytest.skip("no recorded reference counts")
    recs = json.load(open(path))
    graphs = {
        "er4096_d16_s0_l4s2": T.gen_er(4096, 16.0, 0).set_labels(4, 2),
        "chunglu20k_m60k_g2.1_cap600_s1_l4s2": T.gen_chung_lu(20000, 60000, 2.1, 600, 1).set_labels(4, 2),
    }
    dev = {k: T.GraphPreprocessor(csr=v, labeled=True) for k, v in graphs.items()}
    from tests.test_cpu_oracle import SLOW, known_failures
    bad = known_failures()
    for r in recs:
        key = (r["graph"], r["pattern"], r["labeled"])
        P = T.PatternPreprocessor(text=r["text"], labeled=r["labeled"])
        got = T.count(dev[r["graph"]], P).count
        if key in SLOW:  # no pinned count: the result must not depend on the launch shape
            assert got == T.count(dev[r["graph"]], P, T.default_options(merge_window=-1, chunk_cap=128)).count
            continue
        assert got == bad.get(key, r["count"]), r


def test_batch_equals_single_launches(er, cl, T):
    """Many plans of uneven size in one launch (one slot per plan, labeled
    and unlabeled mixed in one call) give the same counts as one launch each."""
    rng = random.Random(11)
    for case in (er, cl):
        texts = [(TRIANGLE, False), (CYCLE4, False), (clique(4), False), (HOUSE, False), (clique(5), False)]
        # labeled random patterns of every size; unlabeled ones stay small
        # (a sparse unlabeled 7-vertex pattern has ~1e12 matches here)
        texts += [(random_pattern(3 + t % 5, 0.5, 4, rng), True) for t in range(10)]
        texts += [(random_pattern(3 + t % 2, 0.6, 4, rng), False) for t in range(4)]
        plans = [T.PatternPreprocessor(text=t, labeled=lab) for t, lab in texts]
        batch, _ = T.count_batch(case.dev, plans)
        assert batch == [T.count(case.dev, p).count for p in plans]


def test_batch_on_edge_ranges(cl, T):
    """Batched slots honour the option's edge range like single launches."""
    plans = [T.PatternPreprocessor(text=t) for t in (TRIANGLE, CYCLE4, clique(4))]
    e = cl.csr.nedges
    parts = [T.count_batch(cl.dev, plans, T.default_options(edge_begin=b, edge_end=min(e, b + e // 3 + 1)))[0]
             for b in range(0, e, e // 3 + 1)]
    whole, _ = T.count_batch(cl.dev, plans)
    assert [sum(p[i] for p in parts) for i in range(3)] == whole


def test_captured_launch_and_autotuned_options(cl_small, T):
    """Launches replayed from a cached CUDA graph, and the autotuner's chosen
    options, both give the counts of the default launch."""
    rng = random.Random(17)
    plans = [T.PatternPreprocessor(text=t) for t in (TRIANGLE, CYCLE4, clique(4), HOUSE)]
    plans += [T.PatternPreprocessor(text=random_pattern(4 + t % 3, 0.5, 4, rng), labeled=True) for t in range(4)]
    want, _ = T.count_batch(cl_small.dev, plans)
    for _ in range(3):  # the first call captures, the others replay
        got, _ = T.count_batch(cl_small.dev, plans, T.default_options(graph_capture=1))
        assert got == want
    best, ms = T.autotune(cl_small.dev, plans, sample_stride=8)
    assert ms > 0 and best.edge_stride == 1
    assert T.count_batch(cl_small.dev, plans, best)[0] == want
    best.graph_capture = 1
    assert T.count_batch(cl_small.dev, plans, best)[0] == want
