"""Autotuner for the cycle's launch form.

For a deck and precision, builds one handle per candidate: each tile (elements
per patch = threads per CTA of the hexa and shell kernels), and for a deck
that can run the persistent shell cycle, each tile both with it and with the
per-phase kernels.  It times a few hundred graph-replayed cycles of each with
CUDA events on the handle's stream.  For a deck with both hexas and shells the
two element kernels are independent launches, so their tiles are chosen apart:
each candidate handle also times its hexa and shell kernels alone
(``ECycle.kernel_times``), the fastest hexa tile and the fastest shell tile are
combined, and that pair is timed whole against the best common tile.  The
fastest form is returned.  Results are cached per (deck name, element count,
precision, GPU) in ``autotune_cache.json`` beside this file.

    python -m openradioss_b200.autotune --workload shell_plate
"""
from __future__ import annotations

import json
import os

from . import abi, decks

CANDIDATES = (64, 128, 256)
CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_cache.json")


def _key(deck, precision, gpu):
    return f"{deck.get('name', 'deck')}|{decks.num_elements(deck)}|{precision}|{gpu}"


def _time_cycles(h, ncycles):
    import torch
    s = torch.cuda.ExternalStream(h.stream())
    h.step(min(ncycles, 64))          # first replay captures the graph
    h.reset()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    h.step(ncycles)
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / ncycles


def tune(deck, precision=abi.OR_PREC_SPLIT, ncycles=256, use_cache=True, device=0, verbose=False):
    """Returns (block_hex, block_shell, persistent, {candidate: ms per cycle});
    persistent is the cfg.persistent value of the fastest form (0: the persistent
    cycle where eligible, -1: the per-phase kernels)."""
    import torch
    from .ecycle import ECycle
    gpu = torch.cuda.get_device_name(device)
    key = _key(deck, precision, gpu)
    cache = {}
    if use_cache and os.path.exists(CACHE):
        try:
            cache = json.load(open(CACHE))
        except (OSError, ValueError):
            cache = {}
    if use_cache and key in cache and "persistent" in cache[key]:
        c = cache[key]
        return c["block_hex"], c["block_shell"], c["persistent"], c["ms_per_cycle"]
    has_hex = any(p["hex"] for p in deck["parts"])
    has_shell = any(p["shell"] for p in deck["parts"])
    mixed = has_hex and has_shell
    timings = {}                          # (hexa tile, shell tile, persistent) -> ms per cycle
    kern = {}                             # tile -> per-kernel microseconds of the phase kernels
    for t in CANDIDATES:
        for pers in (0, -1):
            h = ECycle(deck, precision=precision, device=device, graph=1, block_hex=t, block_shell=t,
                       persistent=pers)
            on = h.persistent_info()[0]
            k = (t, t, 0 if on else -1)
            timings[k] = _time_cycles(h, ncycles)
            if mixed and not on:
                kern[t] = h.kernel_times(reps=16)
            h.close()
            if verbose:
                print(f"tile {t} {'persistent' if on else 'phase kernels'}: {timings[k] * 1e3:.2f} us/cycle",
                      flush=True)
            if not on:
                break                     # no persistent form at this tile: the phase kernels are timed
    if mixed and kern:
        th = min(kern, key=lambda t: kern[t]["hex"])
        ts = min(kern, key=lambda t: kern[t]["shell"])
        if th != ts:                      # the two fastest kernels at different tiles: time the pair
            h = ECycle(deck, precision=precision, device=device, graph=1, block_hex=th, block_shell=ts,
                       persistent=-1)
            timings[(th, ts, -1)] = _time_cycles(h, ncycles)
            h.close()
            if verbose:
                print(f"hexa tile {th}, shell tile {ts}: {timings[(th, ts, -1)] * 1e3:.2f} us/cycle", flush=True)
    best = min(timings, key=timings.get)
    bh = best[0] if has_hex else 256
    bs = best[1] if has_shell else 256

    def name(k):
        base = f"{k[0]}" if k[0] == k[1] else f"h{k[0]}s{k[1]}"
        return base + ("p" if k[2] == 0 else "")
    cache[key] = {"block_hex": bh, "block_shell": bs, "persistent": best[2],
                  "ms_per_cycle": {name(k): v for k, v in timings.items()}}
    try:
        json.dump(cache, open(CACHE, "w"), indent=1, sort_keys=True)
    except OSError:
        pass
    return bh, bs, best[2], cache[key]["ms_per_cycle"]


def main():
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="shell_plate",
                    choices=["shell_plate", "hex_block", "mixed_mesh", "batched_parts"])
    ap.add_argument("--precision", default="split", choices=["split", "fp64"])
    ap.add_argument("--cycles", type=int, default=256)
    a = ap.parse_args()
    from . import build
    build.build()
    fac = {"shell_plate": decks.c2_shell_plate, "hex_block": decks.c1_hex_block,
           "mixed_mesh": decks.c4_mixed_mesh, "batched_parts": decks.c3_batched_parts}[a.workload]
    prec = abi.OR_PREC_SPLIT if a.precision == "split" else abi.OR_PREC_FP64
    print(tune(fac(), prec, a.cycles, use_cache=False, verbose=True))


if __name__ == "__main__":
    main()
