"""Multi-rank split of the level-0 edges (world size 2, gloo, CPU): every
rank counts the chunks shard_options deals it and one all_reduce sums them.
The per-rank counts come from the oracle over exactly the edge ranges the
kernel's ticket arithmetic assigns (shard_edge_ranges)."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.abspath(os.path.join(os.path.dirname(__file__), "..")))
    import torch
    import tdfs_b200 as T
    from oracle import pyoracle as po
    from tests.patterns import CYCLE4

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    g = T.gen_er(2048, 12.0, 7)
    G = po.Graph(g.rowptr.copy(), g.colidx.copy())
    P = po.Plan(CYCLE4, False)
    opt = T.shard_options(rank, world)
    assert opt.edge_stride == world and opt.edge_phase == rank
    mine = sum(po.count(G, P, 1, b, e) for b, e in T.shard_edge_ranges(g.nedges, rank, world))
    t = torch.tensor([mine], dtype=torch.int64)
    dist.all_reduce(t)
    if rank == 0:
        q.put((int(t.item()), po.count(G, P), mine))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_sharded_counts_sum_to_total(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    total, want, part = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert total == want and 0 < part < want


def test_shard_ranges_partition_edges():
    import tdfs_b200 as T
    for n, world in [(100, 3), (65646, 4), (31, 2)]:
        seen = []
        for r in range(world):
            seen += [e for b, en in T.shard_edge_ranges(n, r, world) for e in range(b, en)]
        assert sorted(seen) == list(range(n))


def _bench_rank_main(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.abspath(os.path.join(os.path.dirname(__file__), "..")))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # rank r timed 100 + r ms and counted r + 1, 10 * (r + 1) for two patterns
    t, counts = bench.reduce_over_ranks(dist, 100.0 + rank, [rank + 1, 10 * (rank + 1)], device="cpu")
    q.put((rank, t, counts))
    dist.barrier()
    dist.destroy_process_group()


def test_bench_reduces_max_time_and_summed_counts():
    """The N-rank bench line: the slowest rank's time, every rank's counts."""
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, t, counts in got:  # every rank ends with the same whole-job figures
        assert t == 101.0 and counts == [3, 30]


@pytest.mark.parametrize("chunk", [1, 4, 32])
def test_shard_ranges_partition_any_chunk_and_offset(chunk):
    import tdfs_b200 as T
    for begin, end, world in [(0, 100, 3), (600000, 606000, 4), (17, 31, 2), (5, 6, 8)]:
        seen = []
        for r in range(world):
            seen += [e for b, en in T.shard_edge_ranges(end, r, world, chunk, begin) for e in range(b, en)]
        assert sorted(seen) == list(range(begin, end))


def test_bench_deal_chunk():
    import bench
    assert bench.deal_chunk(6000, 1) == 0            # one rank: the library decides
    assert bench.deal_chunk(6000, 2) == 1            # a 1/1000 slice of the power-law graph
    assert bench.deal_chunk(65646, 2) == 4           # the ER graph of the small configs
    assert bench.deal_chunk(10 ** 9, 8) == 32
