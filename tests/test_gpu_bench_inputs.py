"""The benchmarked inputs themselves, pinned to the CPU oracle (bit-exact u64).

Each bench workload's own graph and patterns, at full size, through the same
entry point and launch options the bench times (tdfs_count_batch, captured
launches).  Where the whole count is beyond the oracle (the power-law and
R-MAT configs), the pins are sub-ranges of the bench's own timed edge slices,
hub edges included."""
import pytest

import bench

pytestmark = pytest.mark.gpu


def _oracle_counts(po, g, pats, rng):
    G = po.Graph(g.rowptr, g.colidx, g.labels if any(lab for _, _, lab in pats) else None)
    return [po.count(G, po.Plan(t, lab), 0, rng[0], rng[1]) for _, t, lab in pats]


def test_c13_step_equals_oracle(T, po):
    """The default bench step: config 1's four unlabeled and config 3's eight
    labeled patterns (tdfs_gen_pattern(6 + i % 2, 0.4, 4, 3000 + i)) over the
    whole labeled ER graph, batched, plain and captured."""
    desc, key, spec, slices = bench.workload("c13")
    g = bench.graph_via_library(T, key)
    pats = [(n, bench.pattern_text(s, T.gen_pattern), lab) for n, s, lab in spec]
    want = _oracle_counts(po, g, pats, (0, g.nedges))
    G = T.GraphPreprocessor(csr=g, labeled=True)
    plans = [T.PatternPreprocessor(text=t, labeled=lab) for _, t, lab in pats]
    assert T.count_batch(G, plans)[0] == want
    for _ in range(3):  # capture, then replays
        assert T.count_batch(G, plans, T.default_options(graph_capture=1))[0] == want
    assert [T.count(G, p).count for p in plans] == want
    # the autotuner's options give the same counts
    best, _ = T.autotune(G, plans, sample_stride=4)
    best.graph_capture = 1
    assert T.count_batch(G, plans, best)[0] == want


@pytest.fixture(scope="module")
def powerlaw(T, po):
    g = bench.graph_via_library(T, "cl")
    return g, T.GraphPreprocessor(csr=g), po.Graph(g.rowptr, g.colidx)


@pytest.mark.parametrize("pattern,rng", [
    ("5-clique", (150000, 156000)),   # a whole timed 1/1000 slice of the bench's c2 steps
    ("5-clique", (0, 150)),           # edges of the 21k-degree hub (vertex 0)
    ("house", (600000, 600060)),      # the start of the c2 sub-record's first house slice
    ("house", (3000000, 3000040)),
])
def test_powerlaw_config_slices(T, po, powerlaw, pattern, rng):
    g, G, O = powerlaw
    text = bench.clique(5) if pattern == "5-clique" else bench.HOUSE
    want = po.count(O, po.Plan(text, False), 0, rng[0], rng[1])
    P = T.PatternPreprocessor(text=text)
    o = T.default_options(edge_begin=rng[0], edge_end=rng[1])
    assert T.count(G, P, o).count == want
    o.graph_capture = 1
    assert T.count_batch(G, [P, P], o)[0] == [want, want]


def test_rmat_config_slices(T, po):
    """The scale-24 R-MAT graph of config 4: the 4-clique over the first of
    the bench's timed 1/500000 slices, the 6-clique over its first 12 edges."""
    g = bench.graph_via_library(T, "rmat")
    _, timed = bench.step_ranges(g.nedges, 500000, 20, 5)
    b, e = timed[0]
    O = po.Graph(g.rowptr, g.colidx)
    G = T.GraphPreprocessor(csr=g)
    for k, rng in ((4, (b, e)), (6, (b, b + 12))):
        text = bench.clique(k)
        want = po.count(O, po.Plan(text, False), 0, *rng)
        got = T.count(G, T.PatternPreprocessor(text=text), T.default_options(edge_begin=rng[0], edge_end=rng[1]))
        assert got.count == want, (k, rng)
