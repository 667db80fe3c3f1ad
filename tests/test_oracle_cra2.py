"""Pins the CPU oracle against the reference engine's own output.

The reference's QA case miniqa/RESTART/cra2 is a steel hat-section rail
(768 BT shells, LAW2 Johnson-Cook, /SHFRA/V4 local frames, 17 edge nodes tied
by a /VEL/TRA rigid link and driven by a 500 t added mass at 5 units/s) run in
two engine runs (to t = 2.5 with the link, restarted to t = 5 without it).
The deck is read in place with openradioss_b200.rad; the reference engine's
listing values (every 100 cycles: TIME, TIME-STEP, the element that sets it,
I-ENERGY, K-ENERGY T, K-ENERGY R, 4 significant digits; and the starter's part
masses) are the committed fixture golden/cra2_listing.json, made by
golden/make_cra2_listing.py.  The oracle must reproduce every printed digit.

The deck is not in this repository: the test is skipped where no reference
checkout is present (OR_REFERENCE_ROOT overrides its location).
"""
import json
import math
import os

import numpy as np
import pytest

from openradioss_b200 import abi, rad

REF = os.environ.get("OR_REFERENCE_ROOT", "/root/reference")
CASE = os.path.join(REF, "qa-tests", "miniqa", "RESTART", "cra2", "data")
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cra2_listing.json")

pytestmark = pytest.mark.skipif(not os.path.isdir(CASE), reason="reference checkout with qa-tests not present")


def printed_match(value, printed, units=0.5):
    """value within ``units`` of the last printed digit of the listing's
    4-significant-digit number (0.5: it rounds to what was printed)."""
    ref = float(printed)
    if ref == 0.0:
        return abs(value) < units * 1e-3
    unit = 10.0 ** (math.floor(math.log10(abs(ref))) - 3)
    return abs(value - ref) <= units * unit * (1.0 + 1e-6)


@pytest.fixture(scope="module")
def gold():
    with open(GOLD) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def cra2():
    sd = rad.StarterDeck(os.path.join(CASE, "CRA2V44_0000.rad"))
    engines = [rad.EngineDeck(os.path.join(CASE, f"CRA2V44_000{k}.rad")) for k in (1, 2)]
    return sd, engines


def test_reader_masses_match_starter_listing(cra2, gold):
    sd, _ = cra2
    deck = rad.to_deck(sd)
    assert np.allclose(rad.part_masses(deck), gold["part_mass"], rtol=1e-12, atol=0)
    assert rad.total_mass(deck) == pytest.approx(gold["total_mass"], rel=1e-12)
    g = deck["parts"][0]["shell"][0]
    assert g["prop"]["npt"] == 3 and g["prop"]["ishfram"] == 2 and g["prop"]["ithk"] == 0


@pytest.mark.parametrize("precision", [abi.OR_PREC_FP64, abi.OR_PREC_SPLIT], ids=["fp64", "split"])
def test_oracle_reproduces_reference_listing(cra2, gold, precision):
    from oracle.oracle import Oracle
    sd, (e1, e2) = cra2
    deck = rad.add_engine(rad.to_deck(sd), e1)
    o = Oracle(deck, precision=precision)
    # FP64: every printed digit.  Split form (FP32 element arithmetic): the last
    # printed digit may move by one
    units = 0.5 if precision == abi.OR_PREC_FP64 else 1.5
    bad = []

    def check(run, line):
        t, e = o.time(), o.energies()
        got = dict(time=t["tt"] - t["dt2"], dt=t["dt2"], ie=e["internal"], ke=e["kinetic"], ker=e["kinetic_rot"])
        for k, v in got.items():
            if not printed_match(v, line[k], units):
                bad.append((run, line["cycle"], k, v, line[k]))
        el = rad.element_id(deck, t["ityptst"], t["neltst"])
        if el != line["element"]:
            bad.append((run, line["cycle"], "element", el, line["element"]))

    for run, (eng, gr) in enumerate(zip((e1, e2), gold["runs"])):
        if run == 1:
            o.set_rlink(0, 0, 0)          # the second engine deck has no /VEL card
        lines = {ln["cycle"]: ln for ln in gr["lines"]}
        n = 0
        while o.time()["tt"] < eng.tstop:
            o.step(1)
            if n in lines:                # the listing's cycle-n line: after the run's (n+1)-th cycle
                check(run, lines.pop(n))
            n += 1
        assert not lines, f"run {run}: listing lines not reached: {sorted(lines)}"
        # the listing counts one more than the cycles run; the second run's
        # cycle-0 line (TIME 2.501) is the state after these n cycles
        assert n + 1 == gr["total_cycles"]
    assert not bad, bad


def test_fixture_agrees_with_ref_extract(gold):
    """data/ref.extract (the QA harness's check values) is the second run's cycle-1800 line."""
    ex = gold["ref_extract"]
    line = [ln for ln in gold["runs"][1]["lines"] if ln["cycle"] == int(ex["CYCLE"])][0]
    for k, key in (("time", "TIME"), ("dt", "TSTEP"), ("ie", "IENERGY"), ("ke", "KENERGYT"), ("ker", "KENERGYR")):
        assert float(line[k]) == pytest.approx(float(ex[key]), rel=1e-9)
