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
