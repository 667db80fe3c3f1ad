"""The hexa path's reference case: miniqa SOLIDES/.../flexion/H101.

Six cantilevers of 1-point hexas (1 to 80 elements, LAW1, Iframe 2, Isolid 1,
Ismstr 4), clamped at one end; each free end is tied to a /RBODY whose main
node carries a constant 40 kN /CLOAD; 848 cycles.  The deck as
openradioss_b200.rad reads it is the fixture golden/h101_deck.* and the
reference's listings are golden/h101_listing.json (golden/make_h101_case.py).

* The starter-equivalent rigid-body initialisation (INIRBY: main node moved to
  the centre of mass, body mass, inertia tensor, principal inertias) reproduces
  every digit the starter listing prints.
* The CPU oracle (element cycle + RBYFOR / RBYVIT / the RBYCOR energy
  correction) runs the same number of cycles as the reference engine and
  stays within these relative distances of every printed engine line, the
  largest measured over the run: time step 1.2e-3, kinetic energy 5e-4,
  rotational kinetic energy and external work 1.5e-3, internal energy 6e-3
  (the internal energy is the hourglass-dominated model's smallest quantity:
  the hourglass dissipation is 17 times larger by cycle 800).  The printed
  digits are not all reproduced: the run drifts from the listing from cycle
  ~200 on (the smallest element time step decreases faster here), a
  difference this restatement has not explained.  The element that sets the
  step is not compared: the undeformed cubes tie, and the reference's SPMD
  run breaks ties by domain.
"""
import json
import math
import os
import sys

import numpy as np
import pytest

from openradioss_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from deck_fixture import load_deck  # noqa: E402


@pytest.fixture(scope="module")
def case():
    deck, extra = load_deck(os.path.join(HERE, "golden", "h101_deck"))
    with open(os.path.join(HERE, "golden", "h101_listing.json")) as f:
        gold = json.load(f)
    return deck, extra, gold


def half_unit(printed):
    """Half a unit of the last printed digit of a listing number."""
    mant = printed.upper().split("E")[0]
    exp = int(printed.upper().split("E")[1]) if "E" in printed.upper() else 0
    decimals = len(mant.split(".")[1]) if "." in mant else 0
    return 0.5 * 10.0 ** (exp - decimals)


def test_rbody_init_matches_starter_listing(case):
    deck, _, gold = case
    p = deck["parts"][0]
    ids = list(p["ids"])
    by_id = {rb["id"]: rb for rb in p["rbodies"]}
    assert len(by_id) == len(gold["rigid_bodies"]) == 6
    for g in gold["rigid_bodies"]:
        rb = by_id[g["id"]]
        m = rb["master"]
        assert ids[m] == g["main_node"]
        for c in range(3):
            assert abs(p["x"][m][c] - float(g["x"][c])) <= half_unit(g["x"][c]) * (1 + 1e-9), (g["id"], c)
            assert abs(rb["tensor"][c][c] - float(g["ixx_iyy_izz"][c])) <= half_unit(g["ixx_iyy_izz"][c]) * 1.000001
            assert abs(rb["rby"][9 + c] - float(g["principal"][c])) <= half_unit(g["principal"][c]) * 1.000001
        assert abs(p["ms"][m] - float(g["mass"])) <= half_unit(g["mass"]) * 1.000001
        assert p["inr"][m] == min(rb["rby"][9:12])


def run_listing(model, deck, extra, gold):
    """Runs the deck to its end time one cycle at a time; returns the worst
    relative distance to the listing per quantity, and the cycle count."""
    lines = {ln["cycle"]: ln for ln in gold["lines"]}
    worst = dict(dt=0.0, ie=0.0, ke=0.0, ker=0.0, wext=0.0)
    n = 0
    while model.time()["tt"] < extra["tstop"]:
        model.step(1)
        if n in lines:
            ln = lines.pop(n)
            t, e = model.time(), model.energies()
            got = dict(dt=t["dt2"], ie=e["internal"], ke=e["kinetic"], ker=e["kinetic_rot"], wext=e["external_work"])
            assert abs(t["tt"] - t["dt2"] - float(ln["time"])) <= 2e-3 * max(float(ln["time"]), 1e-30) + 1e-30
            for k, v in got.items():
                ref = float(ln[k])
                if ref != 0.0:
                    worst[k] = max(worst[k], abs(v - ref) / abs(ref))
                else:
                    assert abs(v) <= half_unit(ln[k]), (n, k, v)
        n += 1
    assert not lines, sorted(lines)
    return worst, n + 1


@pytest.mark.parametrize("precision", [abi.OR_PREC_FP64, abi.OR_PREC_SPLIT], ids=["fp64", "split"])
def test_oracle_against_reference_listing(case, precision):
    from oracle.oracle import Oracle
    deck, extra, gold = case
    worst, ncyc = run_listing(Oracle(deck, precision=precision), deck, extra, gold)
    assert ncyc == gold["total_cycles"] == 848
    assert worst["dt"] < 1.2e-3, worst
    assert worst["ke"] < 5e-4, worst
    assert worst["ker"] < 1.5e-3, worst
    assert worst["wext"] < 1.5e-3, worst
    assert worst["ie"] < 6e-3, worst
