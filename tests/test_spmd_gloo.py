"""Domain decomposition of one mesh (openradioss_b200.spmd), host logic on CPU.

The partition must give every element to exactly one rank, carry the full
nodal masses, number the shared nodes once, and let exactly one rank count
each shared node's kinetic energy.  The exchange is then exercised with two
gloo ranks on CPU: each rank assembles nodal forces of its own elements (a
closed-form stand-in for element forces), packs the partial sums of its halo
nodes, all-gathers them and adds them in rank order, and the assembled field
must equal a one-rank assembly of the whole mesh.
"""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from openradioss_b200 import decks, spmd


def _decks():
    return [decks.c2_shell_plate(n=12, size=0.012), decks.c4_mixed_mesh(nx=3, ny=3, nz=6)]


def _groups(part):
    for gi, g in enumerate(part["hex"]):
        yield ("hex", gi, g["ixs"][:, 1:9] - 1, g["ixs"][:, 10])
    for gi, g in enumerate(part["shell"]):
        yield ("shell", gi, g["ixc"][:, 1:5] - 1, g["ixc"][:, 6])


def test_partition_invariants():
    for deck in _decks():
        P = deck["parts"][0]
        for world in (2, 3):
            doms = spmd.partition(deck, world)
            seen = {}
            touched = np.zeros((world, P["x"].shape[0]), bool)
            for r, d in enumerate(doms):
                sub = d["deck"]["parts"][0]
                ids = d["nodes"]
                assert np.array_equal(sub["ms"], P["ms"][ids])
                assert np.array_equal(sub["x"], P["x"][ids])
                for kind, gi, conn, uid in _groups(sub):
                    for u in uid:
                        key = (kind, gi, int(u))
                        assert key not in seen
                        seen[key] = r
                    touched[r, ids[conn.ravel()]] = True
            assert len(seen) == sum(len(uid) for _, _, _, uid in _groups(P))
            shared = np.nonzero(touched.sum(axis=0) > 1)[0]
            assert all(d["nhalo"] == shared.size for d in doms)
            ke = np.zeros(P["x"].shape[0], int)
            for d in doms:
                g = d["nodes"][d["halo_local"]]
                assert np.array_equal(d["halo_slot"], np.searchsorted(shared, g))   # slot = rank in the shared list
                ke[g] += d["halo_ke"]
            assert np.array_equal(ke[shared], np.ones(shared.size, int))


def _element_forces(kind, gi, uid, width):
    k = np.arange(width)[None, :, None]
    c = np.arange(3)[None, None, :]
    u = uid[:, None, None].astype(np.float64)
    return np.sin(0.37 * u + 1.3 * k + 0.7 * c + (5.0 if kind == "shell" else 0.0) + gi)


def _assemble(part):
    f = np.zeros((part["x"].shape[0], 3))
    for kind, gi, conn, uid in _groups(part):
        fe = _element_forces(kind, gi, uid, conn.shape[1])
        for e in range(conn.shape[0]):
            for k in range(conn.shape[1]):
                f[conn[e, k]] += fe[e, k]
    return f


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, which):
    import torch
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    deck = _decks()[which]
    P = deck["parts"][0]
    d = spmd.partition(deck, world)[rank]
    sub = d["deck"]["parts"][0]
    local = _assemble(sub)                                   # this rank's elements only
    slots = torch.from_numpy(d["halo_slot"].astype(np.int64))
    buf = torch.zeros((d["nhalo"], 3), dtype=torch.float64)
    buf[slots] = torch.from_numpy(local[d["halo_local"]])
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    total = parts[0].clone()
    for r in range(1, world):                                # rank order
        total += parts[r]
    f = local.copy()
    f[d["halo_local"]] = total[slots].numpy()
    # every rank now holds the same force on a shared node; collect one copy per node
    glob = torch.zeros((P["x"].shape[0], 3), dtype=torch.float64)
    counted = np.ones(sub["x"].shape[0], bool)
    counted[d["halo_local"]] = d["halo_ke"].astype(bool)
    glob[torch.from_numpy(d["nodes"][counted])] = torch.from_numpy(f[counted])
    dist.all_reduce(glob)
    if rank == 0:
        ref = _assemble(P)
        err = np.abs(glob.numpy() - ref).max() / np.abs(ref).max()
        assert err < 1e-13, err
    dist.barrier()
    dist.destroy_process_group()


def test_halo_exchange_two_gloo_ranks():
    for which in (0, 1):
        mp.spawn(_worker, args=(2, _free_port(), which), nprocs=2, join=True)
