"""The closed-form count of an independent tail, checked on the CPU.

The match kernel counts the leaves below a node at level s in closed form when
the last t = 2 or 3 pattern vertices have all their backward neighbours at or
above level s and none among themselves (on unlabeled plans also: no order
condition between two of them).  The leaves are then the tuples of distinct
vertices drawn from the tail's candidate sets, counted by inclusion-exclusion
(|A||B| - |A n B|, and for three sets |A||B||C| - |A n B||C| - |A n C||B| -
|B n C||A| + 2|A n B n C|).  This test restates that rule in Python over the
plan the library compiles and checks the resulting totals against the CPU
oracle on small random graphs."""
import random

import numpy as np
import pytest

from tests.golden.make_golden import random_pattern

LESS, LARGER = 0, 1  # condition_order codes of the plan dump (2 = not equal)


def tail_level(plan, labeled):
    k, bn, co = plan["k"], plan["backward_neighbors"], plan["condition_order"]
    for s in range(max(2, k - 4), k - 2):
        ok = all(b <= s for j in range(s + 1, k) for b in bn[j])
        if ok and not labeled:
            ok = all(not (op in (LESS, LARGER) and v > s) for j in range(s + 1, k) for op, v in co[j])
        if ok:
            return s
    return -1


def count_with_tails(rowptr, colidx, labels, plan, labeled):
    """The plan's DFS (the oracle's semantics) with the tail counted in closed form."""
    k, bn, co, L = plan["k"], plan["backward_neighbors"], plan["condition_order"], plan["vertex_labels"]
    n = len(rowptr) - 1
    N = [set(colidx[rowptr[v]:rowptr[v + 1]].tolist()) for v in range(n)]
    s = tail_level(plan, labeled)
    assert s >= 0

    def cands(phi, j):
        c = set.intersection(*[N[phi[b]] for b in bn[j]])
        out = set()
        for x in c:
            if labeled and labels[x] != L[j]:
                continue
            ok = True
            for op, v in co[j]:
                if v >= len(phi):
                    continue
                if labeled or op not in (LESS, LARGER):
                    ok &= x != phi[v]
                elif op == LARGER:
                    ok &= x > phi[v]
                else:
                    ok &= x < phi[v]
            if ok:
                out.add(x)
        return out

    total = 0

    def rec(phi):
        nonlocal total
        level = len(phi) - 1
        if level == s:
            A = [cands(phi, j) for j in range(s + 1, k)]
            if len(A) == 2:
                total += len(A[0]) * len(A[1]) - len(A[0] & A[1])
            else:
                a, b, c = A
                total += (len(a) * len(b) * len(c) - len(a & b) * len(c) - len(a & c) * len(b)
                          - len(b & c) * len(a) + 2 * len(a & b & c))
            return
        for x in cands(phi, level + 1):
            rec(phi + [x])

    orient = plan["orient"] and not labeled  # level-0 edges kept only when u < w
    for u in range(n):
        if labeled and labels[u] != L[0]:
            continue
        for w in cands([u], 1):
            if not orient or u < w:
                rec([u, w])
    return total if labeled else total * plan["multiplicity"]


@pytest.mark.parametrize("labeled", [True, False])
def test_tail_closed_form_equals_enumeration(T, po, labeled):
    g = T.gen_er(60, 7.0, 3).set_labels(2, 4)
    ora = po.Graph(g.rowptr.copy(), g.colidx.copy(), g.labels.copy())
    rowptr, colidx, labels = np.asarray(g.rowptr), np.asarray(g.colidx), np.asarray(g.labels)
    rng = random.Random(21)
    checked = 0
    while checked < 6:
        text = random_pattern(5 + checked % 2, 0.4, 2 if labeled else 1, rng)
        plan = T.PatternPreprocessor(text=text, labeled=labeled).dump()
        if tail_level(plan, labeled) < 0:
            continue
        want = po.count(ora, po.Plan(text, labeled))
        assert count_with_tails(rowptr, colidx, labels, plan, labeled) == want, text
        checked += 1
