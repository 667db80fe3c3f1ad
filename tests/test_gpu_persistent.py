"""The persistent form of step() against the per-phase kernels, bit for bit.

A handle of one shell part without rigid links or loads runs all the cycles of
a step() call in one cooperative launch (openradioss_b200/csrc/
persistent_kernel.cuh).  It performs the same operations in the same order as
the patch and node kernels, so every output must be bitwise equal to a handle
built with OR_ECYCLE_PERSISTENT=0: nodes, element state, energies, time state.
Both forms are also held to the oracle by the parity tests.
"""
import os

import numpy as np
import pytest

from openradioss_b200 import abi, decks

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


def handle(deck, persistent, **kw):
    from openradioss_b200.ecycle import ECycle
    old = os.environ.get("OR_ECYCLE_PERSISTENT")
    os.environ["OR_ECYCLE_PERSISTENT"] = "1" if persistent else "0"
    try:
        h = ECycle(deck, **kw)
    finally:
        if old is None:
            del os.environ["OR_ECYCLE_PERSISTENT"]
        else:
            os.environ["OR_ECYCLE_PERSISTENT"] = old
    assert h.persistent_info()[0] == persistent
    return h


def assert_same(a, b):
    na, nb = a.get_nodes(), b.get_nodes()
    for k in ("x", "d", "v", "vr"):
        assert np.array_equal(na[k], nb[k]), k
    for g in range(len(a.shell_groups)):
        sa, sb = a.shell_state(g), b.shell_state(g)
        for k in sa:
            assert np.array_equal(sa[k], sb[k]), (g, k)
    assert a.energies() == b.energies()
    assert a.time() == b.time()


@pytest.mark.parametrize("precision", [abi.OR_PREC_SPLIT, abi.OR_PREC_FP64], ids=["split", "fp64"])
@pytest.mark.parametrize("tile", [64, 128, 256])
def test_persistent_equals_phase_kernels(lib, precision, tile):
    d = decks.c2_shell_plate(n=40, size=0.04, pressure=4e6)
    p = handle(d, True, precision=precision, block_shell=tile)
    r = handle(d, False, precision=precision, block_shell=tile)
    on, ctas, threads = p.persistent_info()
    assert on and ctas >= 1 and threads % tile == 0 and threads <= 384
    for n in (1, 37, 64, 7):                 # odd and even calls: parity and time carried across
        p.step(n)
        r.step(n)
        assert_same(p, r)


@pytest.mark.parametrize("precision", [abi.OR_PREC_SPLIT, abi.OR_PREC_FP64], ids=["split", "fp64"])
def test_persistent_full_plate(lib, precision):
    """The 200x200 plate of the headline workload (many CTAs, one per SM)."""
    d = decks.c2_shell_plate()
    p = handle(d, True, precision=precision)
    r = handle(d, False, precision=precision)
    assert p.persistent_info()[1] > 64
    p.step(300)
    r.step(300)
    assert_same(p, r)


def test_persistent_generic_points_and_frames(lib):
    """3 integration points (the generic-npt element path, state in memory), the
    /SHFRA/V4 frame, LAW1, and a reset between runs."""
    d = decks.c2_shell_plate(n=24, size=0.024, npt=3, pressure=3e6, law=decks.LAW_ELASTIC)
    d["parts"][0]["shell"][0]["prop"]["ishfram"] = 2
    p = handle(d, True, precision=abi.OR_PREC_SPLIT)
    r = handle(d, False, precision=abi.OR_PREC_SPLIT)
    for _ in range(2):
        p.step(90)
        r.step(90)
        assert_same(p, r)
        p.reset()
        r.reset()


def test_persistent_ineligible_decks_use_phase_kernels(lib):
    from openradioss_b200.ecycle import ECycle
    hexes = ECycle(decks.c1_hex_block(nx=3, ny=3, nz=6))
    assert hexes.persistent_info() == (False, 0, 0)
    eager = ECycle(decks.c2_shell_plate(n=8, size=8e-3), graph=0)
    assert eager.persistent_info()[0] is False
