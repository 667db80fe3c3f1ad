"""The persistent form of step() against the per-phase kernels.

A handle of one shell part without rigid links or loads runs all the cycles of
a step() call in one cooperative launch (openradioss_b200/csrc/
persistent_kernel.cuh).  It performs the same operations in the same order as
the patch and node kernels, so with floating-point contraction off (the
library built with -fmad=false) the nodes, the element state and the time state
are bitwise equal to a handle built with cfg.persistent = -1; the energies,
which the persistent form sums over its cycles per element before summing over
the patch, agree to FP64 rounding (1e-13 relative).  With
FMA contraction (the product build) the compiler may fuse a multiply-add in
one kernel and not in the other; there the two forms are held to the parity
bars against each other and against the oracle.
"""
import numpy as np
import pytest

from openradioss_b200 import abi, decks

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP64_PLASTIC_IP_TOL = 1e-9       # integration-point state of flowing shells (E/H amplification)
SPLIT_TOL = 1e-5


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def libs():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openradioss_b200 import build
    build.build()
    build.build(variant="nofma")
    from openradioss_b200.ecycle import load_library
    return {"fma": load_library(), "nofma": load_library(build.OUT_NOFMA)}


def handle(deck, persistent, lib, **kw):
    from openradioss_b200.ecycle import ECycle
    h = ECycle(deck, lib=lib, persistent=0 if persistent else -1, **kw)
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
    ea, eb = a.energies(), b.energies()
    for k in eb:
        assert abs(ea[k] - eb[k]) <= 1e-13 * abs(eb[k]), (k, ea[k], eb[k])
    assert a.time() == b.time()


def assert_close(a, b, precision):
    """Persistent (a) against per-phase (b), FMA build: the parity bars."""
    na, nb = a.get_nodes(), b.get_nodes()
    if precision == abi.OR_PREC_FP64:
        for k in ("d", "v", "vr"):
            assert rel(na[k], nb[k]) < FP64_TOL, (k, rel(na[k], nb[k]))
        for g in range(len(a.shell_groups)):
            sa, sb = a.shell_state(g), b.shell_state(g)
            for k in ("sig", "pla", "thk", "hourg", "eint"):
                if np.abs(sb[k]).max() > 0:
                    assert rel(sa[k], sb[k]) < FP64_PLASTIC_IP_TOL, (g, k, rel(sa[k], sb[k]))
        ea, eb = a.energies(), b.energies()
        for k in ("internal", "kinetic", "kinetic_rot", "hourglass", "plastic_work"):
            assert abs(ea[k] - eb[k]) <= FP64_TOL * abs(eb[k]) + 1e-300, k
    else:
        assert rel(na["d"], nb["d"]) < SPLIT_TOL, rel(na["d"], nb["d"])
    ta, tb = a.time(), b.time()
    assert ta["ncycle"] == tb["ncycle"]
    tol = FP64_TOL if precision == abi.OR_PREC_FP64 else SPLIT_TOL
    for k in ("tt", "dt2"):
        assert abs(ta[k] - tb[k]) <= tol * tb[k], k


@pytest.mark.parametrize("precision", [abi.OR_PREC_SPLIT, abi.OR_PREC_FP64], ids=["split", "fp64"])
@pytest.mark.parametrize("tile", [64, 128, 256])
def test_persistent_equals_phase_kernels_without_contraction(libs, precision, tile):
    d = decks.c2_shell_plate(n=40, size=0.04, pressure=4e6)
    p = handle(d, True, libs["nofma"], precision=precision, block_shell=tile)
    r = handle(d, False, libs["nofma"], precision=precision, block_shell=tile)
    on, ctas, threads = p.persistent_info()
    assert on and ctas >= 1 and threads % tile == 0 and threads <= 384
    for n in (1, 37, 64, 7):                 # odd and even calls: parity and time carried across
        p.step(n)
        r.step(n)
        assert_same(p, r)


@pytest.mark.parametrize("precision", [abi.OR_PREC_SPLIT, abi.OR_PREC_FP64], ids=["split", "fp64"])
@pytest.mark.parametrize("tile", [64, 128, 256])
def test_persistent_against_phase_kernels_and_oracle(libs, precision, tile):
    """The product build: both forms within the parity bars of each other and of
    the FP64 oracle."""
    from oracle.oracle import Oracle
    d = decks.c2_shell_plate(n=40, size=0.04, pressure=4e6)
    p = handle(d, True, libs["fma"], precision=precision, block_shell=tile)
    r = handle(d, False, libs["fma"], precision=precision, block_shell=tile)
    o = Oracle(d, nthreads=8)
    for n in (1, 37, 64, 7):
        p.step(n)
        r.step(n)
        o.step(n)
        assert_close(p, r, precision)
    on = o.get_nodes()
    tol = FP64_TOL if precision == abi.OR_PREC_FP64 else SPLIT_TOL
    for h in (p, r):
        assert rel(h.get_nodes()["d"], on["d"]) < tol


@pytest.mark.parametrize("precision", [abi.OR_PREC_SPLIT, abi.OR_PREC_FP64], ids=["split", "fp64"])
def test_persistent_full_plate(libs, precision):
    """The 200x200 plate of the headline workload (many CTAs, one per SM), at the
    tile that keeps it in one wave."""
    d = decks.c2_shell_plate()
    for name in ("nofma", "fma"):
        p = handle(d, True, libs[name], precision=precision, block_shell=128)
        r = handle(d, False, libs[name], precision=precision, block_shell=128)
        assert p.persistent_info()[1] > 64
        p.step(300)
        r.step(300)
        if name == "nofma":
            assert_same(p, r)
        else:
            assert_close(p, r, precision)


def test_persistent_generic_points_and_frames(libs):
    """3 integration points (the generic-npt element path, state in memory), the
    /SHFRA/V4 frame, LAW1, and a reset between runs."""
    d = decks.c2_shell_plate(n=24, size=0.024, npt=3, pressure=3e6, law=decks.LAW_ELASTIC)
    d["parts"][0]["shell"][0]["prop"]["ishfram"] = 2
    p = handle(d, True, libs["nofma"], precision=abi.OR_PREC_SPLIT)
    r = handle(d, False, libs["nofma"], precision=abi.OR_PREC_SPLIT)
    for _ in range(2):
        p.step(90)
        r.step(90)
        assert_same(p, r)
        p.reset()
        r.reset()


def test_persistent_ineligible_decks_use_phase_kernels(libs):
    from openradioss_b200.ecycle import ECycle
    hexes = ECycle(decks.c1_hex_block(nx=3, ny=3, nz=6))
    assert hexes.persistent_info() == (False, 0, 0)
    eager = ECycle(decks.c2_shell_plate(n=8, size=8e-3), graph=0)
    assert eager.persistent_info()[0] is False
    off = ECycle(decks.c2_shell_plate(n=8, size=8e-3), persistent=-1)
    assert off.persistent_info()[0] is False
    on = ECycle(decks.c2_shell_plate(n=8, size=8e-3))
    assert on.persistent_info()[0] is True
