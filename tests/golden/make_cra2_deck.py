"""Reads the reference's miniqa RESTART/cra2 decks with openradioss_b200.rad and
saves the resulting deck as the fixture cra2_deck.json + cra2_deck.npz (node
coordinates, connectivity, materials, properties, /BCS, /INIVEL, /ADMAS masses
as the reader lumps them, the first engine run's /VEL/TRA rigid link, and the
two runs' end times), so that the CUDA path can be checked against the
reference listings on a machine without the reference checkout:

    OR_REFERENCE_ROOT=<reference checkout> python tests/golden/make_cra2_deck.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from deck_fixture import save_deck  # noqa: E402
from openradioss_b200 import rad  # noqa: E402


def main():
    ref = os.environ.get("OR_REFERENCE_ROOT")
    if not ref:
        sys.exit("set OR_REFERENCE_ROOT to a reference checkout")
    case = os.path.join(ref, "qa-tests", "miniqa", "RESTART", "cra2", "data")
    sd = rad.StarterDeck(os.path.join(case, "CRA2V44_0000.rad"))
    e1 = rad.EngineDeck(os.path.join(case, "CRA2V44_0001.rad"))
    e2 = rad.EngineDeck(os.path.join(case, "CRA2V44_0002.rad"))
    deck = rad.add_engine(rad.to_deck(sd), e1)
    save_deck(deck, os.path.join(HERE, "cra2_deck"),
              extra=dict(source="qa-tests/miniqa/RESTART/cra2/data (CRA2V44_0000.rad, _0001.rad, _0002.rad)",
                         tstop=[float(e1.tstop), float(e2.tstop)],
                         second_run_rlinks=len(e2.rlinks)))
    print("cra2_deck.json / .npz written")


if __name__ == "__main__":
    main()
