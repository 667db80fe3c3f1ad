"""The CUDA hexa path with rigid bodies on the reference's H101 case (six
1-point hexa cantilevers, LAW1, Iframe 2, tips tied to /RBODY main nodes under
a constant /CLOAD; fixture golden/h101_deck.*, listings golden/h101_listing.json).

* FP64 against the CPU oracle after all 848 cycles: 1e-10 relative on nodal
  displacements, velocities and rotational velocities, element stresses, and
  the internal / kinetic / rotational / hourglass energies and external work.
* Split form against the FP64 oracle: 1e-5 on the displacements.
* Against the reference engine's listing, every printed line, within the
  distances the oracle itself keeps from it (tests/test_oracle_h101.py: time
  step 1.2e-3, kinetic energy 5e-4, rotational kinetic energy and external
  work 1.5e-3, internal energy 6e-3), and the same 848 cycles.
"""
import os
import sys

import numpy as np
import pytest

from openradioss_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
sys.path.insert(0, HERE)
from deck_fixture import load_deck  # noqa: E402

pytestmark = pytest.mark.gpu
FP64_TOL = 1e-10


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


@pytest.fixture(scope="module")
def case():
    import json
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openradioss_b200 import build
    build.build()
    deck, extra = load_deck(os.path.join(HERE, "golden", "h101_deck"))
    with open(os.path.join(HERE, "golden", "h101_listing.json")) as f:
        gold = json.load(f)
    return deck, extra, gold


def test_h101_fp64_matches_oracle(case):
    from openradioss_b200.ecycle import ECycle
    from oracle.oracle import Oracle
    deck, _, gold = case
    g = ECycle(deck, precision=abi.OR_PREC_FP64)
    o = Oracle(deck)
    for n in (1, 99, 300, 448):                  # 848 cycles in four calls
        g.step(n)
        o.step(n)
    a, b = g.get_nodes(), o.get_nodes()
    for k in ("d", "v", "vr"):
        assert rel(a[k], b[k]) < FP64_TOL, (k, rel(a[k], b[k]))
    for gi in range(len(g.hex_groups)):
        assert rel(g.hex_state(gi)["sig"], o.hex_state(gi)["sig"]) < FP64_TOL, gi
    ea, eb = g.energies(), o.energies()
    for k in ("internal", "kinetic", "kinetic_rot", "hourglass", "external_work"):
        assert abs(ea[k] - eb[k]) <= FP64_TOL * abs(eb[k]), (k, ea[k], eb[k])
    assert g.time()["ncycle"] == o.time()["ncycle"] == 848
    assert abs(g.time()["dt2"] - o.time()["dt2"]) <= FP64_TOL * o.time()["dt2"]


def test_h101_split_within_1e5(case):
    from openradioss_b200.ecycle import ECycle
    from oracle.oracle import Oracle
    deck, _, _ = case
    s = ECycle(deck, precision=abi.OR_PREC_SPLIT)
    o = Oracle(deck)
    s.step(848)
    o.step(848)
    assert rel(s.get_nodes()["d"], o.get_nodes()["d"]) < 1e-5


def test_h101_cuda_path_against_reference_listing(case):
    from openradioss_b200.ecycle import ECycle
    from test_oracle_h101 import run_listing
    deck, extra, gold = case
    worst, ncyc = run_listing(ECycle(deck, precision=abi.OR_PREC_FP64), deck, extra, gold)
    assert ncyc == gold["total_cycles"] == 848
    assert worst["dt"] < 1.2e-3, worst
    assert worst["ke"] < 5e-4, worst
    assert worst["ker"] < 1.5e-3, worst
    assert worst["wext"] < 1.5e-3, worst
    assert worst["ie"] < 6e-3, worst
