"""Algorithmic bytes of the element cycle (compulsory unique HBM traffic per
cycle), used for the HBM roofline.

s = element/material real size (4 split, 8 FP64); coordinates and
displacements are always FP64 (8 bytes).

* hexa, per element: r+w of sigma(6), EINT, RHO, VOL, QVIS (10 values),
  read OFF, connectivity 8 x 4 B:  21 s + 32;  LAW2 adds r+w PLA, EPSD: +4 s.
* shell, per element: per integration point r+w of sigma(5) and PLA
  (12 s per point), element r+w of THK, EINT(2), HOURG(3) and read OFF (13 s),
  connectivity 16 B:  npt * 12 s + 13 s + 16   (73 s + 16 for 5 points).
* node, per node: r+w X and D in FP64 (96 B), read BCS code (1 B), r+w V (6 s),
  read MS (s): 97 + 7 s;  a node with rotational DOFs adds r+w VR and read IN
  (7 s).  Force assembly traffic is implementation traffic, not counted.
"""
from __future__ import annotations

import json
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FALLBACK_HBM_GBS = 6650.0


def hex_bytes(s, law):
    return 21 * s + 32 + (4 * s if law == 2 else 0)


def shell_bytes(s, npt):
    return npt * 12 * s + 13 * s + 16


def node_bytes(s, rot):
    return 97 + 7 * s + (7 * s if rot else 0)


def deck_bytes(deck, s):
    """(element bytes, node bytes, number of elements) of one cycle of a deck."""
    import numpy as np
    eb = nb = 0
    nel = 0
    for p in deck["parts"]:
        for g in p["hex"]:
            n = g["ixs"].shape[0]
            eb += n * hex_bytes(s, g["mat"]["law"])
            nel += n
        for g in p["shell"]:
            n = g["ixc"].shape[0]
            eb += n * shell_bytes(s, g["prop"]["npt"])
            nel += n
        rot = np.zeros(p["x"].shape[0], bool)
        for g in p["shell"]:
            rot[g["ixc"][:, 1:5].ravel() - 1] = True
        nb += int(rot.sum()) * node_bytes(s, True) + int((~rot).sum()) * node_bytes(s, False)
    return eb, nb, nel


def measured_peak():
    """(HBM GB/s, source) from MEASURED_PEAKS.json, else the pool fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback (MEASURED_PEAKS.json absent: earlier copy measurement on this GPU pool)"
