"""Domain-decomposed run of one mesh against the one-handle run, on one GPU.

The NCCL path with the exchange captured in a CUDA graph runs as one rank
(NCCL takes one GPU per rank): the capture, the replays and the eager
remainder against the one-handle run, bitwise.

Two and three ranks (processes) each run their share of the elements on the
same GPU through the library's SPMD entry points and exchange the shared
nodes' partial sums with their neighbours (spmd.HaloExchange) over gloo
through host memory, so their kernels never wait on each other.  The
assembled displacements, the energies and the time must match a single
handle on the whole mesh: FP64 at 1e-10 relative (the shared nodes' force
sums are associated by rank instead of by patch), the split form at 1e-5.
"""
import os
import socket

import numpy as np
import pytest

from openradioss_b200 import abi, decks

pytestmark = pytest.mark.gpu


def _deck(which):
    if which == "plate":
        return decks.c2_shell_plate(n=24, size=0.024, pressure=5e6)
    return decks.c4_mixed_mesh(nx=4, ny=4, nz=8)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, which, ncycles, precision, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from openradioss_b200 import spmd
    run = spmd.DomainRun(_deck(which), rank, world, precision=precision, device=0, backend="gloo")
    run.step(ncycles)
    nd = run.get_nodes()
    q.put((rank, nd["ids"], nd["d"], nd["v"], run.h.energies(), run.h.time()))
    dist.barrier()
    run.close()
    dist.destroy_process_group()


def _run(which, ncycles, precision, world=2):
    import multiprocessing as pymp
    ctx = pymp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, which, ncycles, precision, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=600) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return sorted(res, key=lambda r: r[0])


@pytest.mark.parametrize("which,ncycles,precision,tol,world", [
    ("plate", 120, abi.OR_PREC_FP64, 1e-10, 2),
    ("mixed", 80, abi.OR_PREC_FP64, 1e-10, 2),
    ("plate", 120, abi.OR_PREC_SPLIT, 1e-5, 2),
    ("plate", 120, abi.OR_PREC_FP64, 1e-10, 3),
    ("mixed", 80, abi.OR_PREC_SPLIT, 1e-5, 3),
])
def test_domains_match_one_handle(which, ncycles, precision, tol, world):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openradioss_b200 import build
    from openradioss_b200.ecycle import ECycle
    build.build()
    deck = _deck(which)
    ref = ECycle(deck, precision=precision)
    ref.step(ncycles)
    rn = ref.get_nodes()
    res = _run(which, ncycles, precision, world)
    n = deck["parts"][0]["x"].shape[0]
    d = np.full((n, 3), np.nan)
    for rank, ids, dd, vv, e, t in res:
        seen = ~np.isnan(d[ids, 0])
        assert np.array_equal(d[ids][seen], dd[seen])        # shared nodes: same update on every rank
        d[ids] = dd
        # the time steps follow the geometry, which differs from the one-handle run at rounding level
        for k in ("tt", "dt2"):
            assert abs(t[k] - ref.time()[k]) <= tol * ref.time()[k], (k, t[k], ref.time()[k])
        assert t["ncycle"] == ref.time()["ncycle"]
    assert not np.isnan(d).any()
    err = np.abs(d - rn["d"]).max() / np.abs(rn["d"]).max()
    assert err < tol, err
    er = ref.energies()
    for k in ("internal", "kinetic", "kinetic_rot", "hourglass"):
        tot = sum(r[4][k] for r in res)
        assert abs(tot - er[k]) <= 10 * tol * max(abs(er[k]), 1e-30), (k, tot, er[k])


def _nccl_worker(port, which, steps, graph_cycles, precision, q):
    import datetime
    import torch.distributed as dist
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=120))
    from openradioss_b200 import spmd
    run = spmd.DomainRun(_deck(which), 0, 1, precision=precision, device=0, backend="nccl",
                         graph_cycles=graph_cycles)
    for n in steps:
        run.step(n)
    nd = run.get_nodes()
    q.put((nd["d"], nd["v"], run.h.energies(), run.h.time(), run.graph is not None))
    run.close()                       # releases the graph before the process group
    dist.destroy_process_group()


@pytest.mark.parametrize("which,precision", [("plate", abi.OR_PREC_FP64), ("mixed", abi.OR_PREC_SPLIT)])
def test_nccl_exchange_in_a_cuda_graph(which, precision):
    """Steps of 70 and 75 cycles with 32-cycle graphs: capture in the first step,
    two replays per step, eager remainders of even and odd length."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import multiprocessing as pymp
    from openradioss_b200 import build
    from openradioss_b200.ecycle import ECycle
    build.build()
    steps = (70, 75)
    deck = _deck(which)
    ref = ECycle(deck, precision=precision, persistent=-1)      # the domain runs the per-phase kernels
    ref.step(sum(steps))
    rn = ref.get_nodes()
    ctx = pymp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_nccl_worker, args=(_free_port(), which, steps, 32, precision, q))
    p.start()
    d, v, e, t, captured = q.get(timeout=600)
    p.join(timeout=120)
    assert p.exitcode == 0
    assert captured
    assert np.array_equal(d, rn["d"]) and np.array_equal(v, rn["v"])
    assert t == ref.time()
    er = ref.energies()
    for k in ("internal", "kinetic", "kinetic_rot", "hourglass", "plastic_work"):
        assert e[k] == er[k], (k, e[k], er[k])
