"""Pattern texts used across the tests (reference .g format)."""
import json
import os

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

TRIANGLE = "# triangle\nv 0 1\nv 1 1\nv 2 1\ne 0 1 1\ne 0 2 1\ne 1 2 1\n"
CYCLE4 = "# 4-cycle\nv 0 1\nv 1 1\nv 2 1\nv 3 1\ne 0 1 1\ne 1 2 1\ne 2 3 1\ne 0 3 1\n"
HOUSE = ("# house\nv 0 1\nv 1 1\nv 2 1\nv 3 1\nv 4 1\n"
         "e 0 1 1\ne 0 2 1\ne 1 2 1\ne 1 3 1\ne 2 4 1\ne 3 4 1\n")


def clique(k: int) -> str:
    s = f"# K{k}\n" + "".join(f"v {i} 1\n" for i in range(k))
    return s + "".join(f"e {i} {j} 1\n" for i in range(k) for j in range(i + 1, k))


def reference_patterns():
    """The reference's 14 shipped patterns (data/pattern/1.g..14.g), as
    recorded in tests/golden/plans.json."""
    with open(os.path.join(GOLDEN, "plans.json")) as f:
        recs = json.load(f)
    seen, out = set(), []
    for r in recs:
        if r["name"].startswith("ref/") and r["name"] not in seen:
            seen.add(r["name"])
            out.append((r["name"], r["text"]))
    return out


K4 = clique(4)
K5 = clique(5)
