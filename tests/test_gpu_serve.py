"""The continuous-batching server: every query's count is the same whether it
runs alone (one plain launch) or admitted into the running kernel among
others; admission rejects what can never fit; the slot table turns over."""
import random
import threading
import time

import pytest

from tests.golden.make_golden import random_pattern
from tests.patterns import CYCLE4, HOUSE, TRIANGLE, clique

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def graph(T):
    return T.GraphPreprocessor(csr=T.gen_er(4096, 16.0, 0).set_labels(4, 2), labeled=True)


def _queries(T, n, seed, labeled):
    """Random connected queries; labeled ones of 3-7 vertices, unlabeled ones
    of 3-5 (larger sparse unlabeled patterns have ~1e10+ matches here)."""
    rng = random.Random(seed)
    out = []
    for i in range(n):
        k = 3 + rng.randrange(5 if labeled else 3)
        out.append(T.PatternPreprocessor(text=random_pattern(k, rng.uniform(0.3, 0.8), 4, rng), labeled=labeled))
    return out


@pytest.mark.parametrize("labeled", [True, False])
def test_mixed_equals_alone(T, graph, labeled):
    qs = _queries(T, 80, 5 if labeled else 6, labeled)
    alone = [T.count(graph, q).count for q in qs]
    srv = T.Server(graph, labeled=labeled, max_inflight=16)
    # queries arrive while earlier ones are on the device
    tickets = []
    for i, q in enumerate(qs):
        tickets.append(srv.submit(q))
        if i % 10 == 9:
            time.sleep(0.002)
    got = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert [c for c, _ in got] == alone
    assert st["completed"] == len(qs) and st["p99_us"] >= st["p50_us"] > 0


def test_submitters_from_many_threads(T, graph):
    qs = [T.PatternPreprocessor(text=t) for t in (TRIANGLE, CYCLE4, HOUSE, clique(4))] * 10
    alone = {id(q): T.count(graph, q).count for q in qs}
    srv = T.Server(graph, labeled=False, max_inflight=8)
    res = []  # list.append is atomic under the GIL

    def worker(chunk):
        for q in chunk:
            res.append((q, srv.wait(srv.submit(q))[0]))

    th = [threading.Thread(target=worker, args=(qs[i::4],)) for i in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    srv.close()
    assert len(res) == len(qs)
    assert all(c == alone[id(q)] for q, c in res)


def test_admission_rejects_what_cannot_fit(T, graph):
    srv = T.Server(graph, labeled=False, max_k=5)
    with pytest.raises(T.TdfsError) as e:
        srv.submit(T.PatternPreprocessor(text=clique(7)))
    assert e.value.code == 8
    with pytest.raises(T.TdfsError) as e:
        srv.submit(T.PatternPreprocessor(text=TRIANGLE, labeled=True))  # wrong mode
    assert e.value.code == 8
    srv.close()
    tiny = T.Server(graph, labeled=False, mem_budget=1024)
    with pytest.raises(T.TdfsError) as e:
        tiny.submit(T.PatternPreprocessor(text=TRIANGLE))
    assert e.value.code == 8
    tiny.close()


def test_slot_table_turns_over(T, graph):
    """More queries than one table holds: the server closes the spent table,
    lets the kernel drain and opens the next one."""
    p = T.PatternPreprocessor(text=TRIANGLE)
    want = T.count(graph, p).count
    srv = T.Server(graph, labeled=False, max_inflight=512)
    tickets = [srv.submit(p) for _ in range(4500)]
    counts = [srv.wait(t)[0] for t in tickets]
    srv.close()
    assert counts == [want] * len(tickets)


def test_idle_kernel_is_relaunched(T, graph):
    p = T.PatternPreprocessor(text=CYCLE4)
    want = T.count(graph, p).count
    srv = T.Server(graph, labeled=False, idle_exit_ms=5)
    assert srv.wait(srv.submit(p))[0] == want
    time.sleep(0.1)  # the kernel retires when idle
    assert srv.wait(srv.submit(p))[0] == want
    srv.close()
