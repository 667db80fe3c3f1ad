"""Reads the reference's miniqa SOLIDES/nv_elts/poutre_flex/flexion/H101 case
(six 1-point hexa cantilevers of increasing refinement, LAW1, Iframe 2, each
tip tied to a /RBODY whose main node carries a constant /CLOAD) and writes:

* h101_deck.json + .npz: the deck as openradioss_b200.rad reads it (nodes,
  hexas, materials, properties, /BCS, /FUNCT, /CLOAD, the rigid bodies after
  the starter-equivalent initialisation), and the run's end time;
* h101_listing.json: from the starter listing, every rigid body's
  initialisation (main node position, mass, inertia tensor, principal
  inertias, as printed); from the engine listing, every cycle line (CYCLE,
  TIME, TIME-STEP, ELEMENT, I-ENERGY, K-ENERGY T, K-ENERGY R, EXT-WORK, kept as
  printed) and the total number of cycles.

    OR_REFERENCE_ROOT=<reference checkout> python tests/golden/make_h101_case.py
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from deck_fixture import save_deck  # noqa: E402
from openradioss_b200 import rad  # noqa: E402

LINE = re.compile(r"^\s*(\d+)\s+(\S+)\s+(\S+)\s+SOLID\s+(\d+)\s+(\S+)%\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+")


def rbody_init(path):
    out, cur = [], None
    for line in open(path):
        s = line.split()
        if line.strip().startswith("RIGID BODY ID") and len(s) == 4:
            cur = dict(id=int(s[3]))
            out.append(cur)
        elif cur is not None and line.strip().startswith("PRIMARY NODE"):
            cur["main_node"] = int(s[-1])
        elif cur is not None and line.strip().startswith("NEW X,Y,Z"):
            cur["x"] = s[-3:]
        elif cur is not None and line.strip().startswith("NEW MASS"):
            cur["mass"] = s[-1]
        elif cur is not None and line.strip().startswith("NEW INERTIA xx yy zz"):
            cur["ixx_iyy_izz"] = s[-3:]
        elif cur is not None and line.strip().startswith("PRINCIPAL INERTIA"):
            cur["principal"] = s[-3:]
    return [r for r in out if "principal" in r]


def main():
    ref = os.environ.get("OR_REFERENCE_ROOT")
    if not ref:
        raise SystemExit("set OR_REFERENCE_ROOT to a reference checkout")
    case = os.path.join(ref, "qa-tests", "miniqa", "SOLIDES", "nv_elts", "poutre_flex", "flexion", "H101")
    sd = rad.StarterDeck(os.path.join(case, "data", "CONV_ELS_0000.rad"))
    ed = rad.EngineDeck(os.path.join(case, "data", "CONV_ELS_0001.rad"))
    deck = rad.to_deck(sd)
    save_deck(deck, os.path.join(HERE, "h101_deck"),
              extra=dict(source="qa-tests/miniqa/SOLIDES/nv_elts/poutre_flex/flexion/H101/data",
                         tstop=float(ed.tstop)))
    lines, ncyc = [], None
    for line in open(os.path.join(case, "reference", "CONV_ELS_0001.out")):
        m = LINE.match(line)
        if m:
            c, t, dt, el, _err, ie, ke, ker, wext = m.groups()
            lines.append(dict(cycle=int(c), time=t, dt=dt, element=int(el), ie=ie, ke=ke, ker=ker, wext=wext))
        m = re.search(r"TOTAL NUMBER OF CYCLES\s*:\s*(\d+)", line)
        if m:
            ncyc = int(m.group(1))
    data = dict(source="qa-tests/miniqa/SOLIDES/nv_elts/poutre_flex/flexion/H101/reference (OpenRadioss listings)",
                rigid_bodies=rbody_init(os.path.join(case, "reference", "CONV_ELS_0000.out")),
                total_cycles=ncyc, lines=lines)
    with open(os.path.join(HERE, "h101_listing.json"), "w") as f:
        json.dump(data, f, indent=1)
    print(f"h101: {len(data['rigid_bodies'])} rigid bodies, {len(lines)} cycle lines")


if __name__ == "__main__":
    main()
