"""Domain decomposition of one mesh over ranks (one process per GPU).

The reference runs one mesh on several MPI domains: each domain computes the
element forces of its elements, the domains exchange the partial nodal force
sums of the nodes they share (SPMD_EXCH_A, point to point with the neighbouring
domains only) and take the minimum of their element time steps
(SPMD_GLOB_MIN5), and every domain then applies the same nodal update to its
nodes.  Here a rank is one process driving one handle:

- :func:`partition` splits a single-part deck into ``world`` sub-decks of
  contiguous slabs of elements along the longest axis of the part (the same
  split on every rank, no communication), each with the nodes its elements
  touch (full nodal masses and inertias, as assembled for the whole mesh).  A
  rank numbers its shared ("halo") nodes 0.. in ascending global node order and
  lists, per neighbouring rank, the halo slots of the nodes the two share;
- :class:`HaloExchange` moves, each cycle, only the partial sums of the nodes a
  rank shares with each neighbour (one ``all_to_all_single`` whose split sizes
  are zero for every rank that is not a neighbour), lays each neighbour's
  partials into a buffer of its own in this rank's slot numbering, and
  all-reduces the 16-byte time-step reduction (minimum) over all ranks;
- :class:`DomainRun` uploads its rank's sub-deck, declares the halo to the
  library (``or_ecycle_set_halo``) and runs cycles through the library's
  per-cycle SPMD entry points with that exchange, on the handle's CUDA stream
  (NCCL), or through host memory with the gloo backend.  With NCCL, runs of
  ``graph_cycles`` cycles (even) are captured once into a CUDA graph, the
  collectives included, and replayed; the remainder runs eagerly.

A shared node's force is the sum of the partials of the ranks that hold it, in
rank order (a rank that does not hold it adds nothing), so all ranks apply the
same update; the time step is the minimum over ranks.  Only
``ityptst``/``neltst`` differ from a one-handle run (element numbers are local
to a rank).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi, decks


def _groups(part):
    """(kind, group index, 0-based connectivity) of every element group."""
    for gi, g in enumerate(part["hex"]):
        yield "hex", gi, g["ixs"][:, 1:9] - 1
    for gi, g in enumerate(part["shell"]):
        yield "shell", gi, g["ixc"][:, 1:5] - 1


def partition(deck, world):
    """Returns one dict per rank: ``deck`` (the sub-deck), ``nodes`` (global
    part-local ids of the rank's nodes, ascending), ``halo_local``,
    ``halo_slot``, ``halo_ke`` (local node, its slot in this rank's halo
    numbering, 1 if this rank counts the node's kinetic energy), ``nhalo`` (the
    rank's halo size), ``nhalo_global`` (nodes shared by any two ranks),
    ``neighbours`` (ranks sharing nodes with this one, ascending), ``shared``
    (per neighbour: this rank's slots of the nodes the two share, ascending
    global node order, so both ranks list the same nodes in the same order),
    ``rotations`` (1 if the part has shells: moment sums are exchanged too) and
    ``nel``."""
    if len(deck["parts"]) != 1:
        raise ValueError("domain decomposition takes a single-part deck")
    P = deck["parts"][0]
    x = P["x"]
    axis = int(np.argmax(x.max(axis=0) - x.min(axis=0)))
    # every element with its sort key: (centroid along the axis, kind, group, element)
    keys = []
    for kind, gi, conn in _groups(P):
        c = x[conn].mean(axis=1)[:, axis]
        keys += [(c[e], 0 if kind == "hex" else 1, gi, e) for e in range(conn.shape[0])]
    order = sorted(range(len(keys)), key=lambda i: keys[i])
    nel = len(order)
    bounds = [round(r * nel / world) for r in range(world + 1)]
    rank_of = np.empty(nel, np.int64)
    for r in range(world):
        rank_of[order[bounds[r]:bounds[r + 1]]] = r
    sel, i = {}, 0
    for kind, gi, conn in _groups(P):
        sel[(kind, gi)] = rank_of[i:i + conn.shape[0]]
        i += conn.shape[0]
    touched = np.zeros((world, x.shape[0]), bool)
    for kind, gi, conn in _groups(P):
        for q in range(world):
            touched[q, conn[sel[(kind, gi)] == q].ravel()] = True
    is_halo = touched.sum(axis=0) > 1
    first_rank = np.argmax(touched, axis=0)
    out = []
    for r in range(world):
        nodes = np.nonzero(touched[r])[0]
        local = -np.ones(x.shape[0], np.int64)
        local[nodes] = np.arange(nodes.size)
        sub = decks.new_part(x[nodes])
        for k in ("v", "vr", "ms", "inr", "icodt", "icodr"):
            sub[k] = np.ascontiguousarray(P[k][nodes])
        for gi, g in enumerate(P["hex"]):
            m = sel[("hex", gi)] == r
            if m.any():
                d = dict(g)
                d["ixs"] = g["ixs"][m].copy()
                d["ixs"][:, 1:9] = local[d["ixs"][:, 1:9] - 1] + 1
                if g.get("vol0") is not None:
                    d["vol0"] = np.asarray(g["vol0"])[m]
                sub["hex"].append(d)
        for gi, g in enumerate(P["shell"]):
            m = sel[("shell", gi)] == r
            if m.any():
                d = dict(g)
                d["ixc"] = g["ixc"][m].copy()
                d["ixc"][:, 1:5] = local[d["ixc"][:, 1:5] - 1] + 1
                for k in ("thke", "jc_a"):
                    if g.get(k) is not None:
                        d[k] = np.asarray(g[k])[m]
                sub["shell"].append(d)
        mine = nodes[is_halo[nodes]]                      # ascending global order
        neighbours = [q for q in range(world) if q != r and touched[q, mine].any()]
        shared = {q: np.nonzero(touched[q, mine])[0].astype(np.int32) for q in neighbours}
        sd = dict(deck)
        sd["parts"] = [sub]
        out.append(dict(deck=sd, nodes=nodes, halo_local=local[mine].astype(np.int32),
                        halo_slot=np.arange(mine.size, dtype=np.int32),
                        halo_ke=(first_rank[mine] == r).astype(np.int32), nhalo=int(mine.size),
                        nhalo_global=int(is_halo.sum()), neighbours=neighbours, shared=shared,
                        rotations=int(len(P["shell"]) > 0),
                        nel=int(sum(int((v == r).sum()) for v in sel.values()))))
    return out


class HaloExchange:
    """The per-cycle exchange of one rank, on torch tensors of one device.

    Buffer layout (the library's, ``or_ecycle_spmd_buffer_bytes`` each): nhalo
    force sums of 4 reals (x, y, z, unused), nhalo moment sums of 4 reals, the
    rank's time-step reduction (two unsigned 64-bit keys, minimum wins).
    ``bufs`` holds one such buffer per rank in ``views`` (this rank and its
    neighbours, ascending); this rank's own buffer is the one its element pass
    packs (:meth:`own_ptr`), a neighbour's buffer holds, at this rank's slots of
    the nodes the two share, the neighbour's partial sums and zeros elsewhere,
    and its reduction field stays all ones (no candidate).  After
    :meth:`exchange` the own reduction field holds the minimum over all ranks,
    so the node pass, which sums the buffers in order and takes the minimum of
    their reductions, computes the same forces and time step on every rank.

    Only x, y, z of a sum travel, and moment sums only when the part has
    shells; ``sent_reals`` is the count per cycle.
    """

    _SIGN = -(2 ** 63)

    def __init__(self, dom, rank, world, real_dtype, nbytes, device, backend="nccl"):
        import torch
        self.rank, self.world, self.backend = rank, world, backend
        self.views = sorted(set(dom["neighbours"]) | {rank})
        self.own = self.views.index(rank)
        nh = int(dom["nhalo"])
        isz = torch.empty((), dtype=real_dtype).element_size()
        if nbytes % 8 or nbytes != 2 * nh * 4 * isz + 16:
            raise ValueError("exchange buffer size does not match the halo")
        self.nbytes = nbytes
        self.bufs = torch.zeros(len(self.views) * nbytes, dtype=torch.uint8, device=device)
        acc_at = 2 * nh * 4 * isz
        for v in range(len(self.views)):
            if v != self.own:
                self.bufs[v * nbytes + acc_at: (v + 1) * nbytes] = 255
        self.flat = self.bufs.view(real_dtype)
        a0 = (self.own * nbytes + acc_at) // 8
        self.acc = self.bufs.view(torch.int64)[a0:a0 + 2]
        row = nbytes // isz
        nsec = 2 if dom["rotations"] else 1
        src, dst, counts = [], [], [0] * world
        for q in dom["neighbours"]:
            s = np.asarray(dom["shared"][q], np.int64)
            e = (np.arange(nsec)[:, None, None] * nh * 4 + s[None, :, None] * 4 + np.arange(3)[None, None, :]).ravel()
            src.append(self.own * row + e)
            dst.append(self.views.index(q) * row + e)
            counts[q] = int(e.size)
        cat = lambda parts: np.concatenate(parts) if parts else np.zeros(0, np.int64)
        self.src = torch.from_numpy(cat(src)).to(device)
        self.dst = torch.from_numpy(cat(dst)).to(device)
        self.counts = counts
        self.sent_reals = int(sum(counts))
        self.recv = torch.empty(self.sent_reals, dtype=real_dtype, device=device)

    def exchange_warmup(self):
        """The collectives of :meth:`exchange` on scratch copies, so that NCCL's
        communicators exist before a CUDA graph captures them."""
        import torch.distributed as dist
        if self.world > 1:
            dist.all_to_all_single(self.recv.clone(), self.recv.new_zeros(self.sent_reals), self.counts, self.counts)
        dist.all_reduce(self.acc.clone(), op=dist.ReduceOp.MIN)

    def own_ptr(self):
        return self.bufs.data_ptr() + self.own * self.nbytes

    def views_ptr(self):
        return self.bufs.data_ptr()

    def exchange(self):
        """SPMD_EXCH_A (neighbours only) and SPMD_GLOB_MIN5, on the current stream."""
        import torch
        import torch.distributed as dist
        if self.world > 1:
            send = self.flat.index_select(0, self.src)
            if self.backend == "nccl":
                dist.all_to_all_single(self.recv, send, self.counts, self.counts)
                self.flat.index_copy_(0, self.dst, self.recv)
            else:                                  # gloo: through host memory
                rh = torch.empty(self.recv.shape, dtype=self.recv.dtype)
                dist.all_to_all_single(rh, send.cpu(), self.counts, self.counts)
                self.flat.index_copy_(0, self.dst, rh.to(self.flat.device))
        # unsigned minimum through a signed one: flip the top bit both ways
        if self.backend == "nccl":
            self.acc.bitwise_xor_(self._SIGN)
            dist.all_reduce(self.acc, op=dist.ReduceOp.MIN)
            self.acc.bitwise_xor_(self._SIGN)
        else:
            a = self.acc.cpu() ^ self._SIGN
            dist.all_reduce(a, op=dist.ReduceOp.MIN)
            self.acc.copy_(a ^ self._SIGN)


class DomainRun:
    """One rank of a domain-decomposed run: one handle on this rank's GPU."""

    def __init__(self, deck, rank, world, precision=abi.OR_PREC_FP64, device=0, backend="nccl", graph_cycles=32,
                 **cfg_kw):
        import torch
        from .ecycle import ECycle
        if graph_cycles and (graph_cycles < 0 or graph_cycles % 2):
            raise ValueError("graph_cycles must be even (the time buffers alternate by cycle parity)")
        self.rank, self.world, self.backend = rank, world, backend
        self.graph_cycles = int(graph_cycles) if backend == "nccl" else 0
        self.graph = None
        self._comm_ready = False
        self.dom = partition(deck, world)[rank]
        self.h = ECycle(self.dom["deck"], precision=precision, device=device, graph=0, **cfg_kw)
        hl, hs, hk = (np.ascontiguousarray(self.dom[k], np.int32) for k in ("halo_local", "halo_slot", "halo_ke"))
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        self.h._call("set_halo", 0, int(hl.size), ip(hl), ip(hs), ip(hk), int(self.dom["nhalo"]))
        nb = C.c_longlong()
        self.h._call("spmd_buffer_bytes", C.byref(nb))
        self.nbytes = nb.value
        dev = torch.device("cuda", device)
        real = torch.float32 if precision == abi.OR_PREC_SPLIT else torch.float64
        self.xch = HaloExchange(self.dom, rank, world, real, self.nbytes, dev, backend)
        self.stream = torch.cuda.ExternalStream(self.h.stream(), device=dev)

    def _cycle(self):
        """One cycle: element kernels and halo pack, the exchange, node kernel."""
        self.h._call("spmd_elements", C.c_void_p(self.xch.own_ptr()))
        self.xch.exchange()
        self.h._call("spmd_nodes", C.c_void_p(self.xch.views_ptr()), len(self.xch.views))

    def step(self, ncycles):
        """ncycles cycles; the same call, with the same ncycles, on every rank.

        Every step starts at time-buffer parity 0 (``spmd_begin``), and a graph
        holds an even number of cycles, so a replay always starts at parity 0
        and leaves it there; the library's cycle counter advances by the
        (even) captured count during the capture only."""
        import torch
        import torch.distributed as dist
        t = self.h.times
        n = int(ncycles)
        self.h._call("spmd_begin", C.byref(t[0]))
        with torch.cuda.stream(self.stream):
            G = self.graph_cycles
            if G and n >= G:
                if self.graph is None:
                    if not self._comm_ready:       # the communicators exist before a capture
                        self.xch.exchange_warmup()
                        torch.cuda.current_stream().synchronize()
                        self._comm_ready = True
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g, stream=self.stream):
                        for _ in range(G):
                            self._cycle()
                    self.graph = g
                for _ in range(n // G):
                    self.graph.replay()
                n -= (n // G) * G
            for _ in range(n):
                self._cycle()
        self.h._call("spmd_end", C.byref(t[0]))

    def get_nodes(self):
        """This rank's nodes, with their global (part-local) node ids in ``ids``."""
        out = self.h.get_nodes()
        out["ids"] = self.dom["nodes"]
        return out

    def close(self):
        """Releases the graph (it holds NCCL calls: before destroy_process_group)
        and the handle."""
        self.graph = None
        self.h.close()
