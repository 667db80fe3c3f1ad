"""Runs a workload for a few eager cycles (one launch per kernel per cycle, no
CUDA graph) and prints per-phase device times; the command profiled by ncu.

    python -m openradioss_b200.profile_run --workload shell_plate --cycles 20 [--n 600] [--tile 128]
"""
from __future__ import annotations

import argparse
import json

from . import abi, build, decks
from .ecycle import ECycle

FACTORIES = {
    "shell_plate": lambda n: decks.c2_shell_plate(n=n or 200, size=(n or 200) * 1e-3),
    "hex_block": lambda n: decks.c1_hex_block(nx=n or 10, ny=n or 10, nz=4 * (n or 10)),
    "mixed_mesh": lambda n: decks.c4_mixed_mesh(nx=n or 100, ny=n or 100, nz=2 * (n or 100)),
    "batched_parts": lambda n: decks.c3_batched_parts(),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="shell_plate", choices=sorted(FACTORIES))
    ap.add_argument("--n", type=int, default=0, help="mesh size parameter (0 = workload default)")
    ap.add_argument("--cycles", type=int, default=20)
    ap.add_argument("--precision", default="split", choices=["split", "fp64"])
    ap.add_argument("--tile", type=int, default=0, help="elements per patch (0 = library default)")
    a = ap.parse_args()
    build.build()
    d = FACTORIES[a.workload](a.n)
    prec = abi.OR_PREC_SPLIT if a.precision == "split" else abi.OR_PREC_FP64
    tiles = dict(block_hex=a.tile, block_shell=a.tile) if a.tile else {}
    h = ECycle(d, precision=prec, graph=0, **tiles)
    h.step(a.cycles)
    print(json.dumps({"workload": a.workload, "elements": decks.num_elements(d), "cycles": a.cycles,
                      "phase_ms": h.phase_times(), "launches": h.launch_count(), "time": h.time()}))


if __name__ == "__main__":
    main()
