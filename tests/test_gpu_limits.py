"""Device-side limits: the per-pattern work budget and the bounded idle wait.

Nothing here faults or hangs a GPU.  A budget that runs out makes the warps
drop that pattern's subtrees; the launch still completes and reports the
pattern with TDFS_ERR_TIMEOUT.  The wait test launches the kernel over a
slot that nothing can ever complete (a flag that nothing sets), so every
warp's idle wait runs to its bound; the launch then returns TDFS_ERR_TIMEOUT,
and the context stays usable."""
import pytest

from tests.golden.make_golden import random_pattern
from tests.patterns import CYCLE4, HOUSE, TRIANGLE, clique

pytestmark = pytest.mark.gpu

TIMEOUT = 6  # TDFS_ERR_TIMEOUT


@pytest.fixture(scope="module")
def graph(T):
    csr = T.gen_chung_lu(50000, 150000, 2.1, 3000, 1).set_labels(4, 2)
    return csr, T.GraphPreprocessor(csr=csr, labeled=True)


def test_budget_runs_out_and_others_complete(T, graph):
    _, G = graph
    heavy = T.PatternPreprocessor(text=HOUSE)     # many matches: far above a small budget
    light = T.PatternPreprocessor(text=TRIANGLE)
    want_heavy, want_light = T.count(G, heavy).count, T.count(G, light).count
    # about 1e10 work units for the house on this graph, a few million for the triangle
    counts, status, _ = T.count_batch_status(G, [heavy, light, heavy], T.default_options(work_budget=50_000_000))
    assert status == [TIMEOUT, 0, TIMEOUT] and counts[1] == want_light and counts[0] == counts[2] == 0
    with pytest.raises(T.TdfsError) as e:
        T.count(G, heavy, T.default_options(work_budget=2000))
    assert e.value.code == TIMEOUT and "budget" in str(e.value)
    # a budget that is large enough changes nothing
    counts, status, _ = T.count_batch_status(G, [heavy, light], T.default_options(work_budget=10 ** 12))
    assert status == [0, 0] and counts == [want_heavy, want_light]
    # and the context is usable after the abandoned subtrees
    assert T.count(G, heavy).count == want_heavy


def test_budget_with_every_launch_path(T, graph):
    """Captured launches, no stealing and one-edge tickets honour the budget too."""
    _, G = graph
    P = [T.PatternPreprocessor(text=t) for t in (CYCLE4, clique(4))]
    want = [T.count(G, p).count for p in P]
    for opt in ({"graph_capture": 1}, {"steal": 0}, {"edge_chunk": 1, "split_after_us": -1}):
        counts, status, _ = T.count_batch_status(G, P, T.default_options(work_budget=1, **opt))
        assert status == [TIMEOUT, TIMEOUT], opt
        counts, status, _ = T.count_batch_status(G, P, T.default_options(work_budget=10 ** 12, **opt))
        assert status == [0, 0] and counts == want, opt


def test_served_queries_with_a_budget(T, graph):
    """Queries over budget come back with TDFS_ERR_TIMEOUT; every other
    served count equals its plain count."""
    import random
    _, G = graph
    rng = random.Random(41)
    texts = [random_pattern(3 + t % 5, 0.5, 4, rng) for t in range(40)]
    # a labeled 5-star (heavy around the hubs) and a labeled triangle (light)
    texts += ["v 0 1\nv 1 1\nv 2 1\nv 3 1\nv 4 1\ne 0 1 1\ne 0 2 1\ne 1 2 1\ne 0 3 1\ne 0 4 1\n",
              "v 0 3\nv 1 3\nv 2 3\ne 0 1 1\ne 0 2 1\ne 1 2 1\n"]
    plans = [T.PatternPreprocessor(text=t, labeled=True) for t in texts]
    budget = 2_000_000
    plain = T.count_batch_status(G, plans, T.default_options(work_budget=budget))
    srv = T.Server(G, labeled=True, max_inflight=16, work_budget=budget)
    tickets = [srv.submit(p) for p in plans]
    served, aborted = [], 0
    for tk in tickets:
        try:
            served.append(srv.wait(tk)[0])
        except T.TdfsError as e:
            assert e.code == TIMEOUT
            served.append(None)
            aborted += 1
    st = srv.stats()
    srv.close()
    assert st["aborted"] == aborted and st["completed"] == len(plans)
    exact = [T.count(G, p).count for p in plans]
    for s, c in zip(served, exact):
        assert s is None or s == c
    # the budget is per query: the heaviest queries run out, alone or mixed
    assert sum(s is None for s in served) > 0 and sum(st_ == 0 for st_ in plain[1]) > 0


def test_idle_wait_runs_out_to_its_bound(T, graph):
    _, G = graph
    rc, ms = T.selftest_wait_limit(G, 300)
    assert rc == TIMEOUT and 250 <= ms < 5000
    assert T.count(G, T.PatternPreprocessor(text=TRIANGLE)).count > 0  # the context is usable
