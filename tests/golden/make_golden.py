"""Generate the golden fixtures in tests/golden/ from the reference itself.

    python tests/golden/make_golden.py plans --reference <reference checkout>
    python tests/golden/make_golden.py ref-counts   # on a GPU box

(``--reference`` may also come from the TDFS_REFERENCE environment variable;
it is the checkout whose data/pattern/*.g are recorded.)

``plans``: runs the reference's own PatternPreprocessor (src/pattern.h, with
bliss compiled from its sources; see oracle/Makefile target ``ref``) through
oracle/refdump.cpp on the reference's 14 shipped .g patterns, the triangle /
4-cycle / house of the benchmark configs, a few edge-label corner cases and
seeded random connected patterns, in both ulb and lb modes, and stores every
plan field the reference kernel reads -> plans.json.

``ref-counts``: runs the reference's own CUDA build (oracle/_ref/ulb.out,
lb.out, compiled from the reference sources for sm_100a) on small synthetic
graphs and stores the counts it prints -> ref_counts.json.  The graphs are
written in the reference's file format from the seeded generators.  Only
graphs whose maximum degree stays far below the reference's GRAPH_DEGREE=4096
stack row are used, so its candidate sets never overflow.
"""
from __future__ import annotations

import json
import os
import random
import subprocess
import sys
import tempfile

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

def ref_patterns_dir() -> str:
    """data/pattern of the reference checkout named by --reference or the
    TDFS_REFERENCE environment variable."""
    ref = os.environ.get("TDFS_REFERENCE")
    if "--reference" in sys.argv:
        ref = sys.argv[sys.argv.index("--reference") + 1]
    if not ref:
        raise SystemExit("give the reference checkout: --reference <dir> or TDFS_REFERENCE=<dir>")
    return os.path.join(ref, "data", "pattern")

REFBIN = os.path.join(ROOT, "oracle", "_ref")
OUT = os.path.dirname(os.path.abspath(__file__))

TRIANGLE = "# triangle\nv 0 1\nv 1 1\nv 2 1\ne 0 1 1\ne 0 2 1\ne 1 2 1\n"
CYCLE4 = "# 4-cycle 0-1-2-3\nv 0 1\nv 1 1\nv 2 1\nv 3 1\ne 0 1 1\ne 1 2 1\ne 2 3 1\ne 0 3 1\n"
HOUSE = ("# house: 4-cycle 1-3-4-2 plus triangle 0-1-2\nv 0 1\nv 1 1\nv 2 1\nv 3 1\nv 4 1\n"
         "e 0 1 1\ne 0 2 1\ne 1 2 1\ne 1 3 1\ne 2 4 1\ne 3 4 1\n")
# edge labels other than 1: the reference's |Aut| test compares `== 1` rows
# with `!= 0` images (src/pattern.h:286-301)
ODD_LABELS = "# triangle with one edge label 2\nv 0 1\nv 1 1\nv 2 1\ne 0 1 1\ne 0 2 2\ne 1 2 1\n"
ZERO_EDGE = "# path whose extra edge has label 0 (no edge)\nv 0 1\nv 1 1\nv 2 1\ne 0 1 1\ne 1 2 1\ne 0 2 0\n"


def random_pattern(k: int, density: float, nlabels: int, rng: random.Random) -> str:
    """Connected pattern in valid order (i>0 has an earlier neighbour, 2 ~ 1)."""
    edges = set()
    for i in range(1, k):
        j = 1 if i == 2 else rng.randrange(i)
        edges.add((j, i))
    for i in range(k):
        for j in range(i + 1, k):
            if rng.random() < density:
                edges.add((i, j))
    s = "# random\n" + "".join(f"v {i} {rng.randrange(nlabels)}\n" for i in range(k))
    return s + "".join(f"e {a} {b} 1\n" for a, b in sorted(edges))


def refdump(text: str, labeled: bool) -> dict:
    with tempfile.NamedTemporaryFile("w", suffix=".g", delete=False) as f:
        f.write(text)
        path = f.name
    exe = os.path.join(REFBIN, "refdump_lb" if labeled else "refdump_ulb")
    out = subprocess.run([exe, path], capture_output=True, text=True, check=True).stdout
    os.unlink(path)
    line = next(l for l in out.splitlines() if l.startswith("@@PLAN "))
    return json.loads(line[len("@@PLAN "):])


def make_plans():
    cases = []
    for i in range(1, 15):
        with open(os.path.join(ref_patterns_dir(), f"{i}.g")) as f:
            cases.append((f"ref/{i}.g", f.read()))
    cases += [("triangle", TRIANGLE), ("cycle4", CYCLE4), ("house", HOUSE), ("odd_labels", ODD_LABELS),
              ("zero_edge", ZERO_EDGE)]
    rng = random.Random(20240)
    for t in range(120):
        k = 3 + t % 5
        cases.append((f"random/{t}", random_pattern(k, rng.uniform(0.15, 0.9), 4, rng)))
    out = []
    for name, text in cases:
        for labeled in (False, True):
            out.append({"name": name, "labeled": labeled, "text": text, "plan": refdump(text, labeled)})
    with open(os.path.join(OUT, "plans.json"), "w") as f:
        json.dump(out, f, indent=0)
    print(f"wrote {len(out)} plans")


def make_ref_counts():
    import tdfs_b200 as T
    work = tempfile.mkdtemp()
    graphs = []
    g = T.gen_er(4096, 16.0, 0)
    g.set_labels(4, 2)
    prefix = os.path.join(work, "er4096")
    g.write(prefix)
    graphs.append(("er4096_d16_s0_l4s2", prefix, g.max_degree))
    g2 = T.gen_chung_lu(20000, 60000, 2.1, 600, 1)
    g2.set_labels(4, 2)
    prefix2 = os.path.join(work, "cl20k")
    g2.write(prefix2)
    graphs.append(("chunglu20k_m60k_g2.1_cap600_s1_l4s2", prefix2, g2.max_degree))
    # the reference's shipped patterns, as recorded in plans.json (the GPU box
    # has no copy of the reference tree)
    with open(os.path.join(OUT, "plans.json")) as f:
        recorded = json.load(f)
    patterns = []
    for rec in recorded:
        if rec["name"].startswith("ref/") and not rec["labeled"]:
            patterns.append((rec["name"], rec["text"]))
    patterns += [("triangle", TRIANGLE), ("cycle4", CYCLE4), ("house", HOUSE)]
    rng = random.Random(3)
    for t in range(6):
        patterns.append((f"random_labeled/{t}", random_pattern(6 + t % 2, 0.4, 4, rng)))
    out = []
    for gname, prefix, maxdeg in graphs:
        assert maxdeg < 1024, "reference stack rows hold 4096 vertices"
        for pname, text in patterns:
            path = os.path.join(work, pname.replace("/", "_") + ".g")
            with open(path, "w") as f:
                f.write(text)
            for labeled in (False, True):
                exe = os.path.join(REFBIN, "lb.out" if labeled else "ulb.out")
                r = subprocess.run([exe, prefix, path], capture_output=True, text=True, timeout=600)
                lines = [l for l in r.stdout.splitlines() if l.count("\t") == 2]
                if r.returncode != 0 or not lines:
                    raise RuntimeError(f"{exe} {pname}: rc={r.returncode}\nstdout tail: {r.stdout[-600:]}\n"
                                       f"stderr: {r.stderr[-600:]}")
                last = lines[-1]
                _, ms, cnt = last.split("\t")
                out.append({"graph": gname, "pattern": pname, "text": text, "labeled": labeled,
                            "count": int(cnt), "ms": float(ms)})
                print(gname, pname, labeled, cnt, ms, flush=True)
    dest = os.environ.get("GOLDEN_OUT", os.path.join(OUT, "ref_counts.json"))
    with open(dest, "w") as f:
        json.dump(out, f, indent=0)


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "plans"
    make_plans() if what == "plans" else make_ref_counts()
