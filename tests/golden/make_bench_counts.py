"""Generate tests/golden/bench_counts.json on a GPU box.

    python tests/golden/make_bench_counts.py

The counts of the power-law config's bench work: the 5-clique over the whole
graph and the house over the five fixed 1/1000 slices of the c2 sub-record
(bench.C2_HOUSE_SLICES), plus the house and 5-clique over the slices that
`bench.py --workload c2` times at its default step counts.  These are too
large for the CPU oracle, so they come from this engine, and each is pinned
first: the GPU count over a prefix of the same edge range, as long as the
oracle finishes in a few seconds, must equal the oracle's.  The reference
arm of the bench compares the reference build's counts with these numbers.
"""
from __future__ import annotations

import json
import os
import sys

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def main():
    import tdfs_b200 as T
    g = bench.graph_via_library(T, "cl")
    G = T.GraphPreprocessor(csr=g)
    E = g.nedges
    pats = {"5-clique": bench.clique(5), "house": bench.HOUSE}
    plans = {n: T.PatternPreprocessor(text=t) for n, t in pats.items()}

    def count(name, b, e):
        # pin: a prefix of [b, e) against the CPU oracle, then the whole range
        per, _, pre = bench.oracle_pass(g, [(name, pats[name], False)], [(b, e)], budget_s=1.0)
        pb, pe = pre[name]
        got = T.count(G, plans[name], T.default_options(edge_begin=pb, edge_end=pe)).count
        if got != per[name][0]:
            raise SystemExit(f"{name} [{pb},{pe}): GPU {got} != oracle {per[name][0]}")
        return T.count(G, plans[name], T.default_options(edge_begin=b, edge_end=e)).count

    out = {"graph": "Chung-Lu n=1.1M m=3.0M gamma=2.1 cap=30k seed 1, degree-ordered ids", "nedges": E}
    sl = [(j * E // 1000, (j + 1) * E // 1000) for j in bench.C2_HOUSE_SLICES]
    out["c2"] = {"5-clique": count("5-clique", 0, E), "house": [count("house", b, e) for b, e in sl],
                 "house_edge_ranges": sl}
    slices = {}
    for steps in (5, 20):
        _, timed = bench.step_ranges(E, 1000, steps, 3)
        for b, e in timed:
            for name in pats:
                slices.setdefault(name, {})[f"{b},{e}"] = count(name, b, e)
    out["c2_slices"] = slices
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bench_counts.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
