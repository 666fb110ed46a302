#!/usr/bin/env python
"""Benchmark of the subgraph-counting hot path (matches/s).

    python bench.py [--gpus N --steps K --warmup W] [--workload c2] [--impl tdfs|reference]

One step = one full count of every pattern of the workload over the whole
data graph (all level-0 edges), the graph already resident in HBM.  With N
ranks (torchrun, one process per GPU) the level-0 edge chunks are dealt
round-robin over the ranks (strong scaling, one u64 all-reduce per step).

The JSON line reports
  value       matches/s of the device-timed steps (CUDA events, max over ranks)
  e2e         the same metric through the public C ABI with host buffers:
              graph upload from pinned host memory + counts + read-back
  roofline    merge-model algorithmic bytes per match-kernel launch / mean
              launch time, against the measured HBM copy bandwidth
  cpu_baseline the multithreaded CPU oracle on a bounded edge shard
  clocks      nvidia-smi SM clocks and throttle reasons sampled while timing

--impl reference runs the reference's own CUDA build (oracle/_ref/ulb.out,
lb.out, compiled from the reference sources for sm_100a) on the same graph
written in its file format, reading its own kernel timing line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

TRIANGLE = "# triangle\nv 0 1\nv 1 1\nv 2 1\ne 0 1 1\ne 0 2 1\ne 1 2 1\n"
CYCLE4 = "# 4-cycle\nv 0 1\nv 1 1\nv 2 1\nv 3 1\ne 0 1 1\ne 1 2 1\ne 2 3 1\ne 0 3 1\n"
DIAMOND = "# diamond: 4-cycle plus one chord\nv 0 1\nv 1 1\nv 2 1\nv 3 1\ne 0 1 1\ne 0 2 1\ne 0 3 1\ne 1 2 1\ne 1 3 1\n"
HOUSE = ("# house\nv 0 1\nv 1 1\nv 2 1\nv 3 1\nv 4 1\n"
         "e 0 1 1\ne 0 2 1\ne 1 2 1\ne 1 3 1\ne 2 4 1\ne 3 4 1\n")


def clique(k):
    return f"# K{k}\n" + "".join(f"v {i} 1\n" for i in range(k)) + "".join(
        f"e {i} {j} 1\n" for i in range(k) for j in range(i + 1, k))


def workload(name, T):
    """(description dict, host CSR, [(pattern name, text)], labeled)."""
    if name == "c1":
        g = T.gen_er(4096, 16.0, 0)
        pats = [("triangle", TRIANGLE), ("4-cycle", CYCLE4), ("diamond", DIAMOND), ("4-clique", clique(4))]
        return ({"workload": "ER n=4096 avg-degree 16 seed 0; triangle, 4-cycle, diamond, 4-clique"}, g, pats, False)
    if name == "c2":
        g = T.gen_chung_lu(1_100_000, 3_000_000, 2.1, 30_000, 1)
        pats = [("5-clique", clique(5)), ("house", HOUSE)]
        return ({"workload": "Chung-Lu n=1.1M m=3.0M gamma=2.1 cap=30k seed 1, degree-ordered ids; 5-clique, house"},
                g, pats, False)
    if name == "c3":
        g = T.gen_er(4096, 16.0, 0).set_labels(4, 2)
        pats = [(f"labeled-{i}", T.gen_pattern(6 + i % 2, 0.4, 4, 3 * 1000 + i)) for i in range(8)]
        return ({"workload": "ER n=4096 avg-degree 16 seed 0, labels U[0,4) seed 2; 8 random 6-7 vertex labeled "
                             "patterns (density 0.4, seed 3)"}, g, pats, True)
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi SM clock / throttle-reason sampler (200 ms period)."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def cpu_baseline(g, pats, labeled, shard):
    """The CPU oracle (multithreaded DFS, same plan) on 1/shard of the level-0
    edge chunks.  Returns (record, model bytes, matches) of the sample."""
    from oracle import pyoracle as po
    import tdfs_b200 as T
    G = po.Graph(g.rowptr, g.colidx, g.labels if labeled else None)
    threads = os.cpu_count() or 1
    total = byts = 0
    t0 = time.perf_counter()
    for _, text in pats:
        P = po.Plan(text, labeled)
        for b, e in T.shard_edge_ranges(g.nedges, 0, shard):
            c, nb = po.count(G, P, threads, b, e, with_bytes=True)
            total += c
            byts += nb
    dt = time.perf_counter() - t0
    return ({"value": total / dt if dt > 0 else None, "unit": "matches/s", "cores": threads, "kind": "port",
             "sample": f"level-0 edge chunks t % {shard} == 0 (1/{shard} of the edges), every pattern",
             "seconds": round(dt, 2)}, byts, total)


def run_tdfs(args, rank, world, dist):
    import torch
    import tdfs_b200 as T
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    desc, g, pats, labeled = workload(args.workload, T)
    G = T.GraphPreprocessor(csr=g, labeled=labeled, device=dev)
    plans = [(n, T.PatternPreprocessor(text=t, labeled=labeled)) for n, t in pats]
    opt = T.shard_options(rank, world)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step():
        out = []
        for n, p in plans:
            r = T.count(G, p, opt)
            out.append(r)
        return out

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    step_ms, launch_ms, matches = [], [], 0
    torch.cuda.synchronize()
    for s in range(args.steps):
        flush.zero_()  # L2 flush between timed steps (256 MB > 126 MB L2), outside the events
        ev[s][0].record()
        res = step()
        ev[s][1].record()
        launch_ms += [r.kernel_ms for r in res]
        matches += sum(r.count for r in res)
    torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    if dist:
        dist.barrier()
    clk = clocks.stop()
    total_ms = sum(step_ms)
    per_pattern = {n: r.count for (n, _), r in zip(plans, res)}
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        m = torch.tensor([matches] + list(per_pattern.values()), dtype=torch.int64, device="cuda")
        dist.all_reduce(m)
        matches = int(m[0].item())
        per_pattern = {n: int(v) for n, v in zip(per_pattern, m[1:].tolist())}
    value = matches / (total_ms / 1e3)

    # ---- end to end through the C ABI with host buffers ------------------
    rp = torch.from_numpy(np.ascontiguousarray(g.rowptr)).pin_memory()
    ci = torch.from_numpy(np.ascontiguousarray(g.colidx)).pin_memory()
    lb = torch.from_numpy(np.ascontiguousarray(g.labels)).pin_memory() if labeled else None
    h2d = rp.numel() * 8 + ci.numel() * 4 + (lb.numel() * 4 if lb is not None else 0) + sum(len(t) for _, t in pats)
    d2h = 64 * len(pats)  # the launch control block read back per count
    e2e_s, e2e_m = [], 0
    for s in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        Gh = T.GraphPreprocessor(rowptr=rp.numpy(), colidx=ci.numpy(), labels=None if lb is None else lb.numpy(),
                                 labeled=labeled, device=dev)
        ps = [T.PatternPreprocessor(text=t, labeled=labeled) for _, t in pats]
        e2e_m += sum(T.count(Gh, p, opt).count for p in ps)
        Gh.close()
        e2e_s.append(time.perf_counter() - t0)
    e2e_total = sum(e2e_s)
    if dist:
        t = torch.tensor([e2e_total], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
        m = torch.tensor([e2e_m], dtype=torch.int64, device="cuda")
        dist.all_reduce(m)
        e2e_m = int(m.item())

    line = {
        "metric": "matches_per_s", "value": value, "unit": "matches/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32/u64",
        "data": "synthetic (seeded generators of the benchmark config)",
        "config": dict(desc, parallelism=f"level-0 edge chunks round-robin over {world} rank(s)",
                       l2="flushed between timed steps (256 MB write)", counts=per_pattern),
        "e2e": {"value": e2e_m / e2e_total, "unit": "matches/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": 2 * len(pats) * args.steps,
        "clocks": clk,
    }
    return line, launch_ms, (g, pats, labeled)


def run_reference(args, rank, world):
    """The reference's own CUDA build on the same workload."""
    import tdfs_b200 as T
    if rank != 0:
        return None
    exe = os.path.join(ROOT, "oracle", "_ref", "lb.out" if args.workload == "c3" else "ulb.out")
    if not os.path.exists(exe):
        return {"impl": "reference", "unavailable": "oracle/_ref not built (needs the reference sources)"}
    desc, g, pats, labeled = workload(args.workload, T)
    work = tempfile.mkdtemp(prefix="tdfs_ref_")
    prefix = os.path.join(work, "snap.txt")
    g.write(prefix)
    files = []
    for n, t in pats:
        p = os.path.join(work, n + ".g")
        with open(p, "w") as f:
            f.write(t)
        files.append((n, p))

    def step():
        ms, cnt, out = 0.0, 0, {}
        for n, p in files:
            r = subprocess.run([exe, prefix, p], capture_output=True, text=True, timeout=args.ref_timeout)
            last = [l for l in r.stdout.splitlines() if l.count("\t") == 2][-1]
            _, m, c = last.split("\t")
            ms += float(m)
            cnt += int(c)
            out[n] = int(c)
        return ms, cnt, out

    try:
        for _ in range(args.warmup):
            step()
        tot_ms, tot_c = 0.0, 0
        for _ in range(args.steps):
            ms, c, counts = step()
            tot_ms += ms
            tot_c += c
    except subprocess.TimeoutExpired:
        return {"impl": "reference", "unavailable": f"reference build exceeded {args.ref_timeout}s per pattern"}
    value = tot_c / (tot_ms / 1e3)
    return {"impl": "reference", "metric": "matches_per_s", "value": value, "unit": "matches/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot_ms / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32/u64",
            "data": "synthetic", "config": dict(desc, counts=counts, timing="the reference's own cudaEvent pair "
                                                 "around its kernel (cu_test.cu:81-97)"),
            "cpu_baseline": {"value": value, "unit": "matches/s", "cores": 0, "kind": "reference",
                             "sample": "the reference's CUDA build on the GPU (it has no CPU path)"},
            "e2e": {"value": value, "unit": "matches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--impl", default="tdfs", choices=["tdfs", "reference"])
    ap.add_argument("--cpu-shard", type=int, default=0, help="CPU baseline sample: 1/shard of the edge chunks")
    ap.add_argument("--ref-timeout", type=int, default=600)
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl" if args.impl == "tdfs" else "gloo", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if dist:
            dist.destroy_process_group()
        return
    line, launch_ms, (g, pats, labeled) = run_tdfs(args, rank, world, dist)
    if rank == 0:
        peak, kind = measured_hbm_peak()
        shard = args.cpu_shard or {"c1": 1, "c3": 1, "c2": 2000}.get(args.workload, 1000)
        if world == 1:
            cb, model_bytes, sample_matches = cpu_baseline(g, pats, labeled, shard)
            line["cpu_baseline"] = cb
        else:
            line["cpu_baseline"] = None
            model_bytes = sample_matches = 0
        mean_launch_s = statistics.mean(launch_ms) / 1e3 if launch_ms else None
        if sample_matches and mean_launch_s:
            per_match = model_bytes / sample_matches
            per_launch = per_match * line["value"] * (sum(launch_ms) / 1e3) / len(launch_ms)
            achieved = per_launch / mean_launch_s / 1e9
            line["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                "frac": achieved / peak, "peak_kind": kind, "traffic": None,
                                "bytes_model": "reference-plan merge model, bytes per match from the CPU sample"}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
