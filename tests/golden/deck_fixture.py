"""Saves and loads a deck (the dict built by openradioss_b200.decks or
openradioss_b200.rad) as a JSON tree plus one .npz of its arrays, so that a deck
read from reference QA data can travel without the reference checkout.

    save_deck(deck, "tests/golden/cra2_deck")   ->  cra2_deck.json, cra2_deck.npz
    deck = load_deck("tests/golden/cra2_deck")
"""
from __future__ import annotations

import json

import numpy as np


def _flatten(obj, arrays, path):
    if isinstance(obj, np.ndarray):
        key = f"a{len(arrays)}"
        arrays[key] = obj
        return {"__array__": key}
    if isinstance(obj, dict):
        return {k: _flatten(v, arrays, f"{path}/{k}") for k, v in obj.items()}
    if isinstance(obj, (list, tuple)):
        return [_flatten(v, arrays, f"{path}/{i}") for i, v in enumerate(obj)]
    if isinstance(obj, np.generic):
        return obj.item()
    return obj


def _restore(obj, arrays):
    if isinstance(obj, dict):
        if set(obj) == {"__array__"}:
            return arrays[obj["__array__"]]
        return {k: _restore(v, arrays) for k, v in obj.items()}
    if isinstance(obj, list):
        return [_restore(v, arrays) for v in obj]
    return obj


def save_deck(deck, stem, extra=None):
    arrays = {}
    tree = _flatten({"deck": deck, "extra": extra or {}}, arrays, "")
    np.savez_compressed(stem + ".npz", **arrays)
    with open(stem + ".json", "w") as f:
        json.dump(tree, f, indent=1, sort_keys=True)


def load_deck(stem):
    """(deck, extra) as saved."""
    with open(stem + ".json") as f:
        tree = json.load(f)
    with np.load(stem + ".npz", allow_pickle=False) as z:
        arrays = {k: z[k] for k in z.files}
    out = _restore(tree, arrays)
    return out["deck"], out["extra"]
