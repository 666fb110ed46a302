"""tdfs_estimate (host Knuth estimator with degree-power importance sampling)
against exact counts of the CPU oracle: exact where every probe sees the same
tree (a complete graph, one label), within a few standard errors on ER and
power-law graphs, deterministic per seed, and its argument errors."""
import math
import random

import numpy as np
import pytest

from tests.golden.make_golden import random_pattern
from tests.patterns import CYCLE4, HOUSE, TRIANGLE, clique

ARG = 7  # TDFS_ERR_ARG


def complete_graph(T, n, tmp_path):
    """K_n with every vertex labelled 1, in the reference's binary graph files."""
    rowptr = np.arange(0, n * (n - 1) + 1, n - 1, dtype=np.int64)
    colidx = np.array([j for i in range(n) for j in range(n) if j != i], dtype=np.int32)
    prefix = str(tmp_path / "kn")
    with open(prefix + ".meta.txt", "w") as f:
        f.write(f"{n}\n{len(colidx)}\n4\n{n - 1}\n")
    rowptr.tofile(prefix + ".vertex.bin")
    colidx.tofile(prefix + ".edge.bin")
    np.ones(n, np.int32).tofile(prefix + ".label.bin")
    return T.read_csr(prefix, labeled=True)


def test_exact_on_complete_graph_one_label(T, tmp_path):
    g = complete_graph(T, 24, tmp_path)
    for k, text in [(3, TRIANGLE), (4, CYCLE4), (5, HOUSE), (6, clique(6))]:
        r = T.estimate(g, T.PatternPreprocessor(text=text, labeled=True), 64, 1)
        # every probe sees the same tree: 24*23 edges, then 22, 21, ... candidates
        assert r.matches == pytest.approx(math.perm(24, k), rel=1e-9) and r.matches_rse < 1e-9


@pytest.fixture(scope="module")
def er_pair(T, po):
    g = T.gen_er(4096, 16.0, 0).set_labels(4, 2)
    return g, po.Graph(g.rowptr.copy(), g.colidx.copy(), g.labels.copy())


def test_close_to_oracle_on_er(T, po, er_pair):
    g, O = er_pair
    rng = random.Random(41)
    cases = [(TRIANGLE, False), (CYCLE4, False), (HOUSE, False)]
    cases += [(random_pattern(4 + t % 3, 0.2, 4, rng), True) for t in range(6)]
    checked = 0
    for text, lab in cases:
        want = po.count(O, po.Plan(text, lab))
        r = T.estimate(g, T.PatternPreprocessor(text=text, labeled=lab), 20000, 3)
        if want == 0:  # no probe can find a match that does not exist
            assert r.matches == 0
        elif want >= 100:  # (a handful of matches in a large tree is missed by every probe)
            # unbiased: within 5 standard errors, the error itself below 50%
            assert r.matches_rse < 0.5, (text, r.matches_rse)
            assert abs(r.matches - want) <= 5 * r.matches_rse * r.matches, (text, lab, r.matches, want)
            checked += 1
    assert checked >= 4


def test_close_to_oracle_on_power_law(T, po):
    g = T.gen_chung_lu(20000, 60000, 2.1, 600, 1).set_labels(4, 2)
    O = po.Graph(g.rowptr.copy(), g.colidx.copy(), g.labels.copy())
    rng = random.Random(43)
    cases = [(TRIANGLE, False), (CYCLE4, False)]
    cases += [(random_pattern(5 + t % 2, 0.4, 4, rng), True) for t in range(4)]
    for text, lab in cases:
        want = po.count(O, po.Plan(text, lab))
        r = T.estimate(g, T.PatternPreprocessor(text=text, labeled=lab), 8192, 5)
        assert want > 0
        assert abs(math.log10(r.matches / want)) < 0.3, (text, lab, r.matches, want)


def test_deterministic_per_seed_and_errors(T, er_pair):
    g, _ = er_pair
    P = T.PatternPreprocessor(text=HOUSE)
    a, b = T.estimate(g, P, 3000, 9), T.estimate(g, P, 3000, 9)
    assert a.matches == b.matches and a.scanned == b.scanned and list(a.nodes) == list(b.nodes)
    assert a.nodes[1] > 0 and a.scanned > 0
    with pytest.raises(T.TdfsError) as e:
        T.estimate(g, P, 0, 1)
    assert e.value.code == ARG
    unl = T.gen_er(512, 8.0, 1)
    with pytest.raises(T.TdfsError) as e:
        T.estimate(unl, T.PatternPreprocessor(text=TRIANGLE, labeled=True), 10, 1)
    assert e.value.code == ARG


def test_edge_range_estimates_sum_to_whole(T, po):
    """Estimates over level-0 edge ranges are unbiased for the counts over
    those ranges (the oracle counts the same ranges)."""
    g = T.gen_chung_lu(20000, 60000, 2.1, 600, 1)
    O = po.Graph(g.rowptr.copy(), g.colidx.copy(), None)
    P = T.PatternPreprocessor(text=CYCLE4)
    E = g.nedges
    nonzero = 0
    for b, e in ((0, E // 10), (E // 3, E // 3 + 5000), (E // 2, E // 2 + 20000), (E - 4000, E)):
        want = po.count(O, po.Plan(CYCLE4, False), edge_begin=b, edge_end=e)
        r = T.estimate(g, P, 20000, 7, edge_begin=b, edge_end=e)
        if want == 0:
            assert r.matches == 0
        elif want >= 100:  # (a handful of matches in a large tree is missed by every probe)
            assert abs(r.matches - want) <= 5 * r.matches_rse * r.matches, (b, e, r.matches, want)
            nonzero += 1
    assert nonzero >= 2
