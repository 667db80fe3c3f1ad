"""The reference's miniqa RESTART/cra2 case as a check: its deck (fixture
cra2_deck.*, read from the reference's decks by make_cra2_deck.py) and its
engine listings (fixture cra2_listing.json, by make_cra2_listing.py).

run_and_compare(model) drives a handle or the oracle through both engine runs,
one cycle per call, and returns every listing value it misses: TIME,
TIME-STEP, the element that sets the step, I-ENERGY, K-ENERGY T and
K-ENERGY R, every 100 cycles, each printed with 4 significant digits.
"""
import json
import math
import os

from deck_fixture import load_deck

HERE = os.path.dirname(os.path.abspath(__file__))


def load():
    """(deck, extra, gold): the deck after the first engine deck's /VEL card."""
    deck, extra = load_deck(os.path.join(HERE, "cra2_deck"))
    with open(os.path.join(HERE, "cra2_listing.json")) as f:
        gold = json.load(f)
    return deck, extra, gold


def printed_match(value, printed, units=0.5):
    """value within ``units`` of the last printed digit of the listing's
    4-significant-digit number (0.5: it rounds to what was printed)."""
    ref = float(printed)
    if ref == 0.0:
        return abs(value) < units * 1e-3
    unit = 10.0 ** (math.floor(math.log10(abs(ref))) - 3)
    return abs(value - ref) <= units * unit * (1.0 + 1e-6)


def run_and_compare(model, deck, extra, gold, units):
    """Runs both engine runs on `model` (ECycle or Oracle built from `deck`);
    returns (mismatches, lines checked)."""
    from openradioss_b200 import rad
    bad, checked = [], 0
    for run, (tstop, gr) in enumerate(zip(extra["tstop"], gold["runs"])):
        if run == 1:
            model.set_rlink(0, 0, 0)          # the second engine deck has no /VEL card
        lines = {ln["cycle"]: ln for ln in gr["lines"]}
        n = 0
        while model.time()["tt"] < tstop:
            model.step(1)
            if n in lines:                    # the listing's cycle-n line: after the run's (n+1)-th cycle
                line = lines.pop(n)
                t, e = model.time(), model.energies()
                got = dict(time=t["tt"] - t["dt2"], dt=t["dt2"], ie=e["internal"], ke=e["kinetic"],
                           ker=e["kinetic_rot"])
                for k, v in got.items():
                    if not printed_match(v, line[k], units):
                        bad.append((run, line["cycle"], k, v, line[k]))
                el = rad.element_id(deck, t["ityptst"], t["neltst"])
                if el != line["element"]:
                    bad.append((run, line["cycle"], "element", el, line["element"]))
                checked += 1
            n += 1
        if lines:
            bad.append((run, "listing lines not reached", sorted(lines)))
        # the listing counts one more than the cycles run; the second run's
        # cycle-0 line (TIME 2.501) is the state after these n cycles
        if n + 1 != gr["total_cycles"]:
            bad.append((run, "total cycles", n + 1, gr["total_cycles"]))
    return bad, checked
