"""Pins the CPU oracle against the reference engine's own output.

The reference's QA case miniqa/RESTART/cra2 is a steel hat-section rail
(768 BT shells, LAW2 Johnson-Cook, /SHFRA/V4 local frames, 17 edge nodes tied
by a /VEL/TRA rigid link and driven by a 500 t added mass at 5 units/s) run in
two engine runs (to t = 2.5 with the link, restarted to t = 5 without it).
The deck, as openradioss_b200.rad reads it, is the fixture golden/cra2_deck.*
(golden/make_cra2_deck.py); the reference engine's listing values (every 100
cycles: TIME, TIME-STEP, the element that sets it, I-ENERGY, K-ENERGY T,
K-ENERGY R, 4 significant digits; and the starter's part masses) are the
fixture golden/cra2_listing.json (golden/make_cra2_listing.py).  The oracle
must reproduce every printed digit.

Where a reference checkout is given (OR_REFERENCE_ROOT), the fixture deck is
also checked against a fresh read of the reference's decks.
"""
import os
import sys

import numpy as np
import pytest

from openradioss_b200 import abi, rad

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import cra2_case  # noqa: E402


@pytest.fixture(scope="module")
def case():
    return cra2_case.load()


def test_reader_masses_match_starter_listing(case):
    deck, _, gold = case
    assert np.allclose(rad.part_masses(deck), gold["part_mass"], rtol=1e-12, atol=0)
    assert rad.total_mass(deck) == pytest.approx(gold["total_mass"], rel=1e-12)
    g = deck["parts"][0]["shell"][0]
    assert g["prop"]["npt"] == 3 and g["prop"]["ishfram"] == 2 and g["prop"]["ithk"] == 0


@pytest.mark.parametrize("precision", [abi.OR_PREC_FP64, abi.OR_PREC_SPLIT], ids=["fp64", "split"])
def test_oracle_reproduces_reference_listing(case, precision):
    from oracle.oracle import Oracle
    deck, extra, gold = case
    o = Oracle(deck, precision=precision)
    # FP64: every printed digit.  Split form (FP32 element arithmetic): the last
    # printed digit may move by one
    units = 0.5 if precision == abi.OR_PREC_FP64 else 1.5
    bad, checked = cra2_case.run_and_compare(o, deck, extra, gold, units)
    assert checked == sum(len(r["lines"]) for r in gold["runs"])
    assert not bad, bad


def test_fixture_agrees_with_ref_extract(case):
    """data/ref.extract (the QA harness's check values) is the second run's cycle-1800 line."""
    gold = case[2]
    ex = gold["ref_extract"]
    line = [ln for ln in gold["runs"][1]["lines"] if ln["cycle"] == int(ex["CYCLE"])][0]
    for k, key in (("time", "TIME"), ("dt", "TSTEP"), ("ie", "IENERGY"), ("ke", "KENERGYT"), ("ker", "KENERGYR")):
        assert float(line[k]) == pytest.approx(float(ex[key]), rel=1e-9)


@pytest.mark.skipif(not os.environ.get("OR_REFERENCE_ROOT"), reason="OR_REFERENCE_ROOT not set")
def test_fixture_deck_is_the_reference_deck(case):
    deck, extra, _ = case
    data = os.path.join(os.environ["OR_REFERENCE_ROOT"], "qa-tests", "miniqa", "RESTART", "cra2", "data")
    sd = rad.StarterDeck(os.path.join(data, "CRA2V44_0000.rad"))
    e1 = rad.EngineDeck(os.path.join(data, "CRA2V44_0001.rad"))
    e2 = rad.EngineDeck(os.path.join(data, "CRA2V44_0002.rad"))
    fresh = rad.add_engine(rad.to_deck(sd), e1)
    assert extra["tstop"] == [e1.tstop, e2.tstop]
    p, q = deck["parts"][0], fresh["parts"][0]
    for k in ("x", "v", "ms", "inr", "icodt", "icodr", "ids"):
        assert np.array_equal(p[k], q[k]), k
    for g, h in zip(p["shell"], q["shell"]):
        assert np.array_equal(g["ixc"], h["ixc"]) and np.array_equal(g["thke"], h["thke"])
        assert g["mat"] == h["mat"] and g["prop"] == h["prop"]
    assert all(np.array_equal(a["nodes"], b["nodes"]) for a, b in zip(p["rlinks"], q["rlinks"]))
