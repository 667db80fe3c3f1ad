"""Parity of the shell formulations Ishell 2, 3, 4 and of one-point shells on
the sm_100a path against the CPU oracle.

The device element (ecycle_kernels.cuh shell_element) and the oracle
(oracle/ecycle_oracle.cpp shell_element) both restate CDEFO3's IHBE branches
(cdefo3.F:103-216), CHVIS3 (chvis3.F), CHSTI3 with its yield-stress bound
(chsti3.F), MHVIS3 for one integration point (mhvis3.F) and CFINT3's warping
moments (cfint3.F:208-214).  Each formulation runs on a jittered LAW2 plate
that yields (and on LAW1 for CHSTI3's unbounded branch), through the
persistent kernel and through the per-phase kernels:

* FP64: nodes, time and energies at 1e-10 relative, integration-point state at
  the plastic-flow bar of the other parity tests (1e-9);
* split: nodal displacements within 1e-5 of the split oracle.
"""
import numpy as np
import pytest

from openradioss_b200 import abi, decks

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP64_PLASTIC_IP_TOL = 1e-9
SPLIT_TOL = 1e-5


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def lib():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openradioss_b200 import build
    build.build()
    from openradioss_b200.ecycle import load_library
    return load_library()


def plate(ishell, npt, law=decks.LAW_JOHNSON_COOK):
    d = decks.c2_shell_plate(n=20, size=0.02, pressure=5e6 if law == decks.LAW_JOHNSON_COOK else 2e6,
                             npt=npt, ishell=ishell, law=law)
    pr = d["parts"][0]["shell"][0]["prop"]
    if npt == 1:
        pr["shf"] = 0.0
        pr["dn"] = 0.015
    return d


def run_pair(deck, ncycles, precision, persistent):
    from openradioss_b200.ecycle import ECycle
    from oracle.oracle import Oracle
    g = ECycle(deck, precision=precision, persistent=persistent)
    o = Oracle(deck, precision=precision, nthreads=8)
    g.step(ncycles)
    o.step(ncycles)
    return g, o


CASES = [(2, 5), (3, 5), (4, 5), (3, 3), (4, 3), (1, 1), (3, 1), (4, 1)]


@pytest.mark.parametrize("persistent", [0, -1], ids=["persistent", "phase"])
@pytest.mark.parametrize("ishell,npt", CASES)
def test_formulation_fp64_against_oracle(lib, ishell, npt, persistent):
    d = plate(ishell, npt)
    g, o = run_pair(d, 300, abi.OR_PREC_FP64, persistent)
    if persistent == 0:
        assert g.persistent_info()[0]
    assert o.shell_state(0)["pla"].max() > 0              # plastic flow happened
    a, b = g.get_nodes(), o.get_nodes()
    for k in ("d", "v", "vr"):
        assert rel(a[k], b[k]) < FP64_TOL, (k, rel(a[k], b[k]))
    sa, sb = g.shell_state(0), o.shell_state(0)
    for k in ("sig", "pla", "thk", "hourg", "eint"):
        if np.abs(sb[k]).max() > 0:
            assert rel(sa[k], sb[k]) < FP64_PLASTIC_IP_TOL, (k, rel(sa[k], sb[k]))
    ea, eb = g.energies(), o.energies()
    for k in ("internal", "kinetic", "kinetic_rot", "hourglass", "plastic_work"):
        if abs(eb[k]) > 0:
            assert abs(ea[k] - eb[k]) <= FP64_TOL * abs(eb[k]), (k, ea[k], eb[k])
    ta, tb = g.time(), o.time()
    assert ta["ncycle"] == tb["ncycle"]
    assert abs(ta["tt"] - tb["tt"]) <= FP64_TOL * tb["tt"]


@pytest.mark.parametrize("ishell,npt", [(3, 5), (4, 3), (3, 1)])
def test_formulation_split_against_split_oracle(lib, ishell, npt):
    d = plate(ishell, npt)
    g, o = run_pair(d, 200, abi.OR_PREC_SPLIT, 0)
    assert rel(g.get_nodes()["d"], o.get_nodes()["d"]) < SPLIT_TOL


def test_chsti3_with_law1_is_unbounded(lib):
    """LAW1 leaves SIGY at EP30 (ccoor3.F:126): CHSTI3 without its bound."""
    d = plate(3, 5, law=decks.LAW_ELASTIC)
    g, o = run_pair(d, 250, abi.OR_PREC_FP64, 0)
    assert rel(g.get_nodes()["d"], o.get_nodes()["d"]) < FP64_TOL
    assert rel(g.shell_state(0)["hourg"], o.shell_state(0)["hourg"]) < FP64_TOL


@pytest.mark.parametrize("ishell,npt", [(3, 5), (1, 1)])
def test_adjoint_refuses_other_formulations(lib, ishell, npt):
    from openradioss_b200.ecycle import ECycle, ECycleError
    g = ECycle(plate(ishell, npt), precision=abi.OR_PREC_FP64)
    with pytest.raises(ECycleError) as ei:
        g.adjoint(10, node=5, comp=2, w_disp=1.0, w_plastic=0.0)
    assert ei.value.code == abi.OR_E_UNSUPPORTED
