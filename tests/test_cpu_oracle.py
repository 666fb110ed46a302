"""The oracle pinned against the reference: plan fields against the
reference's own PatternPreprocessor (tests/golden/plans.json), counts against
closed forms on complete graphs and against exhaustive enumeration."""
import json
import math
import os
import random

import numpy as np
import pytest

from tests.patterns import CYCLE4, HOUSE, TRIANGLE, clique, reference_patterns

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _plans():
    with open(os.path.join(GOLDEN, "plans.json")) as f:
        return json.load(f)


def same_plan(ref: dict, got: dict):
    for key, val in ref.items():
        if key == "backward_neighbors_sh":
            for i, dep in enumerate(ref["shared_lvl"]):
                if dep != -1:
                    assert got[key][i] == val[i], (key, i)
        else:
            assert got[key] == val, key


def test_oracle_plans_match_reference(po):
    recs = _plans()
    assert len(recs) >= 250
    for r in recs:
        same_plan(r["plan"], po.Plan(r["text"], r["labeled"]).as_dict())


@pytest.mark.parametrize("name,conds,aut", [
    ("triangle", [[0, 1], [0, 2], [1, 2]], 6),
    ("cycle4", [[0, 1], [0, 2], [0, 3], [1, 3]], 8),
    ("house", [[1, 2]], 2),
    ("ref/1.g", [[0, 1], [2, 3]], 4),
    ("ref/2.g", [[a, b] for a in range(4) for b in range(a + 1, 4)], 24),
    ("ref/7.g", [[a, b] for a in range(5) for b in range(a + 1, 5)], 120),
    ("ref/5.g", [[1, 2], [1, 3], [1, 4], [2, 4]], 8),
])
def test_plan_known_answers(po, name, conds, aut):
    """Conditions and |Aut| printed by the reference preprocessor."""
    rec = next(r for r in _plans() if r["name"] == name and not r["labeled"])
    d = po.Plan(rec["text"], False).as_dict()
    assert d["conditions"] == conds
    assert d["multiplicity"] == aut


def complete_graph(n):
    rowptr = np.arange(0, n * (n - 1) + 1, n - 1, dtype=np.int64)
    colidx = np.array([j for i in range(n) for j in range(n) if j != i], dtype=np.int32)
    return rowptr, colidx


@pytest.mark.parametrize("n", [6, 8, 11])
def test_oracle_closed_forms_on_complete_graphs(po, n):
    rowptr, colidx = complete_graph(n)
    G = po.Graph(rowptr, colidx, np.ones(n, np.int32))
    for text in [TRIANGLE, CYCLE4, HOUSE, clique(4), clique(5)] + [t for _, t in reference_patterns()[:7]]:
        k = sum(1 for l in text.splitlines() if l.startswith("v"))
        want = math.perm(n, k)
        assert po.count(G, po.Plan(text, False), threads=2) == want
        assert po.count(G, po.Plan(text, True), threads=2) == want  # one label everywhere


def test_oracle_matches_bruteforce(po):
    rng = random.Random(11)
    from tests.golden.make_golden import random_pattern
    for trial in range(40):
        n = rng.randint(6, 10)
        edges = {(i, j) for i in range(n) for j in range(i + 1, n) if rng.random() < rng.uniform(0.3, 0.8)}
        adj = [[] for _ in range(n)]
        for i, j in edges:
            adj[i].append(j)
            adj[j].append(i)
        rowptr = np.cumsum([0] + [len(a) for a in adj]).astype(np.int64)
        colidx = np.array([v for a in adj for v in sorted(a)], dtype=np.int32)
        labels = np.array([rng.randrange(2) for _ in range(n)], np.int32)
        G = po.Graph(rowptr, colidx, labels)
        for labeled in (False, True):
            P = po.Plan(random_pattern(rng.randint(3, 5), rng.uniform(0.3, 0.9), 2, rng), labeled)
            assert po.count(G, P, threads=2) == po.bruteforce(G, P)


def test_oracle_rejects_bad_patterns(po):
    with pytest.raises(po.OracleError):
        po.Plan("v 0 1\nv 1 1\nv 2 1\ne 0 1 1\n", False)  # vertex 2 has no earlier neighbour
    with pytest.raises(po.OracleError):
        po.Plan("v 0 1\nv 1 1\ne 0 1 1\n", False)  # fewer than 3 vertices


def _graph_from_name(T, name):
    if name == "er4096_d16_s0_l4s2":
        return T.gen_er(4096, 16.0, 0).set_labels(4, 2)
    if name == "chunglu20k_m60k_g2.1_cap600_s1_l4s2":
        return T.gen_chung_lu(20000, 60000, 2.1, 600, 1).set_labels(4, 2)
    raise KeyError(name)


def known_failures():
    with open(os.path.join(GOLDEN, "ref_known_failures.json")) as f:
        return {(c["graph"], c["pattern"], c["labeled"]): c["expected"] for c in json.load(f)["cases"]}


# unlabeled 6-7 vertex random patterns on the power-law graph: 1e9-1e10
# matches, hours of CPU-oracle time, so no pinned expectation is recorded;
# the reference's own count is unreliable there (its labeled counterparts
# are recorded failures) and the GPU covers them by option invariance
SLOW = {("chunglu20k_m60k_g2.1_cap600_s1_l4s2", f"random_labeled/{t}", False) for t in range(6)}


def test_oracle_matches_reference_build(T, po):
    """The oracle reproduces every count the reference's own CUDA build
    printed (tests/golden/ref_counts.json), except the recorded reference
    failures, where it gives the expected count instead."""
    recs = json.load(open(os.path.join(GOLDEN, "ref_counts.json")))
    bad = known_failures()
    graphs = {}
    checked = 0
    for r in recs:
        key = (r["graph"], r["pattern"], r["labeled"])
        if key in SLOW:
            continue
        if r["graph"] not in graphs:
            c = _graph_from_name(T, r["graph"])
            graphs[r["graph"]] = po.Graph(c.rowptr.copy(), c.colidx.copy(), c.labels.copy())
        got = po.count(graphs[r["graph"]], po.Plan(r["text"], r["labeled"]))
        if key in bad:
            assert got == bad[key] and got != r["count"], key
        else:
            assert got == r["count"], key
        checked += 1
    assert checked >= 80


def test_reference_failure_independent_recount(T):
    """The ER case the reference miscounts, recounted by a plain Python
    enumeration of injective edge-preserving maps (no plan, no symmetry)."""
    recs = json.load(open(os.path.join(GOLDEN, "ref_counts.json")))
    r = next(x for x in recs if x["graph"] == "er4096_d16_s0_l4s2" and x["pattern"] == "random_labeled/0"
             and not x["labeled"])
    g = T.gen_er(4096, 16.0, 0)
    adj = [set(g.colidx[g.rowptr[v]:g.rowptr[v + 1]].tolist()) for v in range(g.n)]
    lines = r["text"].splitlines()
    k = sum(1 for l in lines if l.startswith("v"))
    edges = [tuple(map(int, l.split()[1:3])) for l in lines if l.startswith("e")]
    nbr = {i: {b if a == i else a for a, b in edges if i in (a, b)} for i in range(k)}
    # the count does not depend on the enumeration order: place the most
    # constrained vertex next (most placed neighbours, then highest degree)
    order = [max(range(k), key=lambda v: len(nbr[v]))]
    while len(order) < k:
        order.append(max((v for v in range(k) if v not in order),
                         key=lambda v: (len(nbr[v] & set(order)), len(nbr[v]))))
    back = [[order.index(u) for u in nbr[order[i]] if order.index(u) < i] for i in range(k)]

    def rec(i, phi):
        cand = set.intersection(*[adj[phi[j]] for j in back[i]])
        if i == k - 1:  # the last vertex: count, do not recurse
            return len(cand.difference(phi))
        return sum(rec(i + 1, phi + [x]) for x in cand if x not in phi)

    total = sum(rec(2, [u, v]) for u in range(g.n) for v in adj[u])
    assert total == known_failures()[("er4096_d16_s0_l4s2", "random_labeled/0", False)] != r["count"]
