"""Pins the CUDA path (through the C-ABI) against the reference engine's own
output: the miniqa RESTART/cra2 rail (768 BT shells, LAW2 with a yield cap,
3 integration points, /SHFRA/V4 frames, a rigid link released between the two
engine runs, 3,375 cycles) from the fixture golden/cra2_deck.*, compared with
every line of the reference listings (golden/cra2_listing.json): TIME,
TIME-STEP, the element that sets the step, I-ENERGY, K-ENERGY T and
K-ENERGY R, 4 significant digits.

Bars: FP64 reproduces every printed digit (within half a unit of the last
digit); the split form stays within one unit of what the rounding printed
(1.5 units of the last digit), as the CPU oracle test requires.
"""
import os
import sys

import pytest

from openradioss_b200 import abi

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import cra2_case  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openradioss_b200 import build
    build.build()
    from openradioss_b200.ecycle import load_library
    return load_library()


@pytest.mark.parametrize("precision", [abi.OR_PREC_FP64, abi.OR_PREC_SPLIT], ids=["fp64", "split"])
def test_cuda_path_reproduces_reference_listing(lib, precision):
    from openradioss_b200.ecycle import ECycle
    deck, extra, gold = cra2_case.load()
    h = ECycle(deck, precision=precision)
    units = 0.5 if precision == abi.OR_PREC_FP64 else 1.5
    bad, checked = cra2_case.run_and_compare(h, deck, extra, gold, units)
    assert checked == sum(len(r["lines"]) for r in gold["runs"]) == 35
    assert not bad, bad
