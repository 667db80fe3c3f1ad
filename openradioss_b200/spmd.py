"""Domain decomposition of one mesh over ranks (one process per GPU).

The reference runs one mesh on several MPI domains: each domain computes the
element forces of its elements, the domains exchange the partial nodal force
sums of the nodes they share (SPMD_EXCH_A) and take the minimum of their
element time steps (SPMD_GLOB_MIN5), and every domain then applies the same
nodal update to its nodes.  Here a rank is one process driving one handle:

- :func:`partition` splits a single-part deck into ``world`` sub-decks of
  contiguous slabs of elements along the longest axis of the part (the same
  split on every rank, no communication), each with the nodes its elements
  touch (full nodal masses and inertias, as assembled for the whole mesh), and
  numbers the shared ("halo") nodes in ascending global node order;
- :class:`DomainRun` uploads its rank's sub-deck, declares the halo to the
  library (``or_ecycle_set_halo``) and runs cycles through the library's
  per-cycle SPMD entry points, exchanging the halo buffers with
  ``torch.distributed.all_gather_into_tensor`` on the handle's CUDA stream
  (NCCL), or through host memory with the gloo backend.  With NCCL, runs of
  ``graph_cycles`` cycles (even) are captured once into a CUDA graph, the
  collective included, and replayed; the remainder runs eagerly.

A shared node's force is the sum of every rank's partial in rank order, so all
ranks apply the same update; the time step is the minimum over ranks.  Only
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
    ``halo_slot``, ``halo_ke`` (local node, global halo slot, 1 if this rank
    counts the node's kinetic energy), ``nhalo`` and ``nel``."""
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
    halo_nodes = np.nonzero(touched.sum(axis=0) > 1)[0]
    slot_of = -np.ones(x.shape[0], np.int64)
    slot_of[halo_nodes] = np.arange(halo_nodes.size)
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
        mine = nodes[slot_of[nodes] >= 0]
        sd = dict(deck)
        sd["parts"] = [sub]
        out.append(dict(deck=sd, nodes=nodes, halo_local=local[mine].astype(np.int32),
                        halo_slot=slot_of[mine].astype(np.int32),
                        halo_ke=(first_rank[mine] == r).astype(np.int32), nhalo=int(halo_nodes.size),
                        nel=int(sum(int((v == r).sum()) for v in sel.values()))))
    return out


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
        self.buf = torch.zeros(self.nbytes, dtype=torch.uint8, device=dev)
        self.bufs = torch.zeros(world * self.nbytes, dtype=torch.uint8, device=dev)
        self.stream = torch.cuda.ExternalStream(self.h.stream(), device=dev)

    def _cycle(self):
        """One cycle: element kernels and halo pack, the exchange, node kernel."""
        import torch
        import torch.distributed as dist
        self.h._call("spmd_elements", C.c_void_p(self.buf.data_ptr()))
        if self.backend == "nccl":
            dist.all_gather_into_tensor(self.bufs, self.buf)
        else:
            host = self.buf.cpu()          # waits for this cycle's element kernels
            parts = [torch.empty_like(host) for _ in range(self.world)]
            dist.all_gather(parts, host)
            self.bufs.copy_(torch.cat(parts))
        self.h._call("spmd_nodes", C.c_void_p(self.bufs.data_ptr()), self.world)

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
                    if not self._comm_ready:       # the communicator exists before a capture
                        dist.all_gather_into_tensor(self.bufs, self.buf)
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
