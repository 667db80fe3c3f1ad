"""Multi-rank sharding of independent parts, exercised with gloo on CPU.

Each of two ranks computes the assignment locally, runs its parts through the
CPU oracle, and the ranks exchange (part index, final displacement norm) over
gloo; the union must cover every part exactly once and match a single-rank run.
"""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from openradioss_b200 import decks, shard


def test_assignment_balanced_and_complete():
    sizes = [5, 100, 7, 60, 60, 3, 40]
    a = shard.assign_parts(sizes, 3)
    assert sorted(sum(a, [])) == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in r) for r in a]
    assert max(loads) - min(loads) <= max(sizes)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch
    from oracle.oracle import Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    d = decks.c3_batched_parts(nparts=5, seed=11, scale=0.005)
    mine = shard.assign_parts(shard.part_sizes(d), world)[rank]
    sub = shard.rank_deck(d, rank, world)
    o = Oracle(sub)
    o.step(20)
    res = torch.zeros(len(d["parts"]), dtype=torch.float64)
    cnt = torch.zeros(len(d["parts"]), dtype=torch.float64)
    for k, pi in enumerate(mine):
        res[pi] = float(np.linalg.norm(o.get_nodes(k)["d"]))
        cnt[pi] = 1
    dist.all_reduce(res)
    dist.all_reduce(cnt)
    if rank == 0:
        out.put((res.numpy().tolist(), cnt.numpy().tolist()))
    dist.destroy_process_group()


def test_two_rank_shards_match_single_rank():
    from oracle.oracle import Oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res, cnt = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert cnt == [1.0] * len(cnt)
    d = decks.c3_batched_parts(nparts=5, seed=11, scale=0.005)
    o = Oracle(d)
    o.step(20)
    ref = [float(np.linalg.norm(o.get_nodes(k)["d"])) for k in range(len(d["parts"]))]
    np.testing.assert_allclose(res, ref, rtol=0, atol=0)
