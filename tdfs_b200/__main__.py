"""Command line: count patterns on a graph file or a seeded synthetic graph.

    python -m tdfs_b200 count --graph PREFIX|er:N,DEG,SEED|cl:N,M,GAMMA,CAP,SEED|rmat:SCALE,EF,SEED
                              --pattern FILE.g|triangle|cycle4|diamond|house|k4|k5|k6|k7|gen:K,DENSITY,NLABELS,SEED
                              [--pattern ...] [--labels NLABELS,SEED] [--labeled] [--reps R]
                              [--edges BEGIN,END] [--opt name=value ...]

With one pattern, prints one line per repetition: pattern, kernel ms, count
(the ulb/lb line).  With several, they run as one batched launch
(tdfs_count_batch) and each repetition prints "batch", the kernel ms and the
counts.  `gen:` patterns come from tdfs_gen_pattern.
"""
from __future__ import annotations

import argparse
import sys

import tdfs_b200 as T

NAMED = {
    "triangle": "v 0 1\nv 1 1\nv 2 1\ne 0 1 1\ne 0 2 1\ne 1 2 1\n",
    "cycle4": "v 0 1\nv 1 1\nv 2 1\nv 3 1\ne 0 1 1\ne 1 2 1\ne 2 3 1\ne 0 3 1\n",
    "diamond": "v 0 1\nv 1 1\nv 2 1\nv 3 1\ne 0 1 1\ne 0 2 1\ne 0 3 1\ne 1 2 1\ne 1 3 1\n",
    "house": "v 0 1\nv 1 1\nv 2 1\nv 3 1\nv 4 1\ne 0 1 1\ne 0 2 1\ne 1 2 1\ne 1 3 1\ne 2 4 1\ne 3 4 1\n",
}
for _k in range(4, 8):
    NAMED[f"k{_k}"] = "".join(f"v {i} 1\n" for i in range(_k)) + "".join(
        f"e {i} {j} 1\n" for i in range(_k) for j in range(i + 1, _k))


def load_graph(spec: str, labels: str | None, labeled: bool):
    kind, _, args = spec.partition(":")
    a = args.split(",") if args else []
    if kind == "er":
        csr = T.gen_er(int(a[0]), float(a[1]), int(a[2]))
    elif kind == "cl":
        csr = T.gen_chung_lu(int(a[0]), int(a[1]), float(a[2]), int(a[3]), int(a[4]))
    elif kind == "rmat":
        csr = T.gen_rmat(int(a[0]), int(a[1]), 0.57, 0.19, 0.19, int(a[2]))
    else:
        return T.GraphPreprocessor(spec, labeled=labeled)
    if labels:
        nl, seed = (int(x) for x in labels.split(","))
        csr.set_labels(nl, seed)
    return T.GraphPreprocessor(csr=csr, labeled=labeled)


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m tdfs_b200")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("count")
    c.add_argument("--graph", required=True)
    c.add_argument("--pattern", required=True, action="append")
    c.add_argument("--labels")
    c.add_argument("--labeled", action="store_true")
    c.add_argument("--reps", type=int, default=1)
    c.add_argument("--edges")
    c.add_argument("--opt", action="append", default=[])
    args = ap.parse_args(argv)
    g = load_graph(args.graph, args.labels, args.labeled)
    plans = []
    for spec in args.pattern:
        if spec in NAMED:
            plans.append(T.PatternPreprocessor(text=NAMED[spec], labeled=args.labeled))
        elif spec.startswith("gen:"):
            k, d, nl, seed = spec[4:].split(",")
            plans.append(T.PatternPreprocessor(text=T.gen_pattern(int(k), float(d), int(nl), int(seed)),
                                               labeled=args.labeled))
        else:
            plans.append(T.PatternPreprocessor(spec, labeled=args.labeled))
    kw = {}
    for o in args.opt:
        k, v = o.split("=")
        kw[k] = int(v)
    if args.edges:
        b, e = args.edges.split(",")
        kw["edge_begin"], kw["edge_end"] = int(b), int(e)
    opt = T.default_options(**kw)
    for _ in range(args.reps):
        if len(plans) == 1:
            r = T.count(g, plans[0], opt)
            print(f"{args.pattern[0]}\t{r.kernel_ms:f}\t{r.count}", flush=True)
        else:
            counts, ms = T.count_batch(g, plans, opt)
            print("batch\t%f\t%s" % (ms, " ".join(str(c) for c in counts)), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
