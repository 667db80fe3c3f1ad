"""The launch-form autotuner (openradioss_b200/autotune.py) on small decks.

A mixed hexa + shell deck has no persistent form; its hexa and shell tiles are
chosen apart from the per-kernel times, and the returned pair is the fastest of
the forms timed.  A one-part shell plate is timed with and without the
persistent shell cycle.
"""
import pytest

from openradioss_b200 import abi, decks

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def autotune():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openradioss_b200 import autotune as at, build
    build.build()
    return at


def key(bh, bs, pers):
    return (f"{bh}" if bh == bs else f"h{bh}s{bs}") + ("p" if pers == 0 else "")


def test_mixed_deck_tiles_chosen_apart(autotune):
    d = decks.c4_mixed_mesh(nx=8, ny=8, nz=16, ncycles=64)
    bh, bs, pers, ms = autotune.tune(d, abi.OR_PREC_SPLIT, ncycles=64, use_cache=False)
    assert bh in autotune.CANDIDATES and bs in autotune.CANDIDATES
    assert pers == -1                                   # no persistent form with hexas
    for t in autotune.CANDIDATES:                       # every common tile was timed
        assert f"{t}" in ms and ms[f"{t}"] > 0
    assert ms[key(bh, bs, pers)] == min(ms.values())


def test_shell_plate_times_both_forms(autotune):
    d = decks.c2_shell_plate(n=40, size=0.04, ncycles=64)
    bh, bs, pers, ms = autotune.tune(d, abi.OR_PREC_SPLIT, ncycles=64, use_cache=False)
    assert pers in (0, -1)
    assert any(k.endswith("p") for k in ms)             # the persistent cycle was timed
    assert any(not k.endswith("p") for k in ms)         # and the per-phase kernels
    assert ms[key(bs, bs, pers)] == min(ms.values())
