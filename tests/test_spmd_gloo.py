"""Domain decomposition of one mesh (openradioss_b200.spmd), host logic on CPU.

The partition must give every element to exactly one rank, carry the full
nodal masses, number each rank's shared nodes in ascending global order, list
for every pair of neighbouring ranks the same shared nodes in the same order,
and let exactly one rank count each shared node's kinetic energy.

The exchange (spmd.HaloExchange, the code the GPU ranks run) is then exercised
with two and three gloo ranks on CPU, on buffers in the library's layout: each
rank assembles nodal forces and moments of its own elements (a closed-form
stand-in for element forces), packs the partial sums of its halo nodes and a
time-step reduction, exchanges with its neighbours only, and sums the buffers
as the node pass does.  The assembled field must equal a one-rank assembly of
the whole mesh, be the same bit for bit on every rank holding a node and equal
to an all-gather of every rank's buffer summed in rank order, the reduction
must be the unsigned minimum over all ranks, and a rank must send only the
partials of the nodes it shares with each neighbour.
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
        for world in (2, 3, 4):
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
            ke = np.zeros(P["x"].shape[0], int)
            for r, d in enumerate(doms):
                assert d["nhalo_global"] == shared.size
                g = d["nodes"][d["halo_local"]]
                assert np.array_equal(g, np.intersect1d(d["nodes"], shared))       # ascending global order
                assert np.array_equal(d["halo_slot"], np.arange(d["nhalo"]))
                ke[g] += d["halo_ke"]
                assert d["neighbours"] == [q for q in range(world) if q != r and touched[q, g].any()]
                for q in d["neighbours"]:
                    mine = g[d["shared"][q]]
                    theirs = doms[q]["nodes"][doms[q]["halo_local"][doms[q]["shared"][r]]]
                    assert np.array_equal(mine, theirs)
                    assert np.array_equal(mine, np.nonzero(touched[r] & touched[q])[0])
            assert np.array_equal(ke[shared], np.ones(shared.size, int))
            if world > 2:                                # slabs: a rank's neighbours are the adjacent slabs
                assert all(len(d["neighbours"]) <= 2 for d in doms)


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


def _pack(d, f, m, acc, real):
    """This rank's buffer in the library's layout: forces, moments, reduction."""
    import torch
    nh = d["nhalo"]
    isz = torch.empty((), dtype=real).element_size()
    nbytes = 2 * nh * 4 * isz + 16
    fm = np.zeros((2, nh, 4))
    fm[0, :, :3] = f[d["halo_local"]]
    fm[1, :, :3] = m[d["halo_local"]]
    buf = torch.zeros(nbytes, dtype=torch.uint8)
    buf[:2 * nh * 4 * isz] = torch.from_numpy(fm.ravel()).to(real).view(torch.uint8)
    buf[2 * nh * 4 * isz:] = torch.tensor(acc, dtype=torch.int64).view(torch.uint8)
    return buf, nbytes


def _node_sums(bufs, nview, nh, real):
    """What the node pass computes from the buffers: per slot, the buffers' sums
    in order (the first one assigned, the others added); the minimum reduction."""
    import torch
    isz = torch.empty((), dtype=real).element_size()
    nbytes = bufs.numel() // nview
    tot, acc = None, None
    for v in range(nview):
        b = bufs[v * nbytes:(v + 1) * nbytes]
        fm = b[:2 * nh * 4 * isz].view(real).view(2, nh, 4)[:, :, :3].clone()
        a = [int(x) & (2 ** 64 - 1) for x in b[2 * nh * 4 * isz:].view(torch.int64)]
        tot = fm if tot is None else tot + fm
        acc = a if acc is None else [min(p, q) for p, q in zip(acc, a)]
    return tot, acc


def _acc_of(rank):
    """Reductions with the top bit set on some ranks: the minimum is unsigned."""
    big = [2 ** 63 + 5 + rank, 2 ** 64 - 1 - rank]
    small = [1000 + 7 * rank, 2 ** 62 + rank]
    return [v - 2 ** 64 if v >= 2 ** 63 else v for v in (small if rank == 1 else big)]


def _worker(rank, world, port, which, real_name):
    import torch
    real = getattr(torch, real_name)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    deck = _decks()[which]
    P = deck["parts"][0]
    doms = spmd.partition(deck, world)
    d = doms[rank]
    sub = d["deck"]["parts"][0]
    f = _assemble(sub)                                       # this rank's elements only
    m = np.cos(f)                                            # moment partials: any per-rank field
    buf, nbytes = _pack(d, f, m, _acc_of(rank), real)
    xch = spmd.HaloExchange(d, rank, world, real, nbytes, torch.device("cpu"), backend="gloo")
    own = xch.bufs[xch.own * nbytes:(xch.own + 1) * nbytes]
    own.copy_(buf)
    xch.exchange()
    tot, acc = _node_sums(xch.bufs, len(xch.views), d["nhalo"], real)
    # the reduction: the unsigned minimum over all ranks
    want = [min(int(x) & (2 ** 64 - 1) for x in col) for col in zip(*(_acc_of(r) for r in range(world)))]
    assert acc == want
    # only shared nodes' partials leave the rank, moments too (shells in the part)
    nsec = 2 if d["rotations"] else 1
    assert xch.sent_reals == sum(3 * nsec * len(d["shared"][q]) for q in d["neighbours"])
    assert set(q for q in range(world) if xch.counts[q]) == set(d["neighbours"])
    # against an all-gather of every rank's buffer in the global halo numbering,
    # summed in rank order: bit for bit
    g_nodes = d["nodes"][d["halo_local"]]
    shared_all = sorted(set().union(*(set(e["nodes"][e["halo_local"]].tolist()) for e in doms)))
    pos = {n: i for i, n in enumerate(shared_all)}
    gl = torch.zeros((2, len(shared_all), 3), dtype=real)
    gl[0, [pos[n] for n in g_nodes]] = torch.from_numpy(f[d["halo_local"]]).to(real)
    gl[1, [pos[n] for n in g_nodes]] = torch.from_numpy(m[d["halo_local"]]).to(real)
    parts = [torch.empty_like(gl) for _ in range(world)]
    dist.all_gather(parts, gl)
    ag = parts[0].clone()
    for r in range(1, world):
        ag += parts[r]
    assert torch.equal(tot, ag[:, [pos[n] for n in g_nodes]])
    # one copy of every node's assembled force, to compare with one rank on the whole mesh
    fl = f.copy()
    fl[d["halo_local"]] = tot[0].double().numpy()
    glob = torch.zeros((P["x"].shape[0], 3), dtype=torch.float64)
    counted = np.ones(sub["x"].shape[0], bool)
    counted[d["halo_local"]] = d["halo_ke"].astype(bool)
    glob[torch.from_numpy(d["nodes"][counted])] = torch.from_numpy(fl[counted])
    dist.all_reduce(glob)
    if rank == 0:
        ref = _assemble(P)
        err = np.abs(glob.numpy() - ref).max() / np.abs(ref).max()
        assert err < (1e-13 if real == torch.float64 else 1e-6), err
    dist.barrier()
    dist.destroy_process_group()


def test_halo_exchange_gloo_ranks():
    for world in (2, 3):
        for which in (0, 1):
            for real in ("float64", "float32"):
                mp.spawn(_worker, args=(world, _free_port(), which, real), nprocs=world, join=True)
