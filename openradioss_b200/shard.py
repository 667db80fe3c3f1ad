"""Sharding of independent parts across ranks (one process per GPU).

Parts of a batched deck are independent units (each keeps its own time step),
so a multi-GPU run assigns whole parts to ranks with no data-path collective:
largest-first greedy on element count, ties broken by part index, which gives
the same assignment on every rank without communication.  A single-part deck
is replicated (each rank runs its own copy: weak scaling).
"""
from __future__ import annotations

import heapq

from . import decks


def part_sizes(deck):
    return [decks.num_elements(dict(parts=[p])) for p in deck["parts"]]


def assign_parts(sizes, world):
    """Returns one list of part indices per rank."""
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + sizes[i], r))
    return [sorted(x) for x in out]


def rank_deck(deck, rank, world):
    """The sub-deck a rank runs: its parts (several parts) or the whole deck
    (single part, replicated)."""
    if len(deck["parts"]) <= 1 or world == 1:
        return deck
    mine = assign_parts(part_sizes(deck), world)[rank]
    sub = dict(deck)
    sub["parts"] = [deck["parts"][i] for i in mine]
    return sub
