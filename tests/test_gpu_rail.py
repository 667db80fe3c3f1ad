"""Parity of the sm_100a path on a crash rail: /SHFRA/V4 element frames
(ISHFRAM 2), 3-point LAW2 shells with a yield cap, and a /VEL/TRA rigid
link carrying an added mass (openradioss_b200.decks.hat_rail), against the CPU
oracle.  The oracle itself reproduces the reference engine's listing of the QA
case miniqa/RESTART/cra2, which uses the same features (test_oracle_cra2.py).

Tolerances as in test_gpu_parity.py: plain FP64 1e-10 normwise on nodal
displacements, velocities, energies and time; 1e-9 on integration-point state
of plastically flowing shells; split form 1e-5 on displacements against the
FP64 oracle.
"""
import ctypes as C

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


def compare(g, o, tol_nodes, tol_ip):
    a, b = g.get_nodes(), o.get_nodes()
    for k in ("d", "v", "vr"):
        assert rel(a[k], b[k]) < tol_nodes, (k, rel(a[k], b[k]))
    ta, tb = g.time(), o.time()
    assert ta["ncycle"] == tb["ncycle"]
    assert abs(ta["tt"] - tb["tt"]) <= tol_nodes * tb["tt"]
    assert abs(ta["dt2"] - tb["dt2"]) <= tol_nodes * tb["dt2"]
    ea, eb = g.energies(), o.energies()
    for k in ("internal", "kinetic", "kinetic_rot", "hourglass", "plastic_work"):
        assert abs(ea[k] - eb[k]) <= tol_nodes * max(abs(eb[k]), 1e-300), (k, ea[k], eb[k])
    if tol_ip is not None:
        sa, sb = g.shell_state(0), o.shell_state(0)
        for k in ("sig", "pla", "thk", "hourg", "eint"):
            assert rel(sa[k], sb[k]) < tol_ip, (k, rel(sa[k], sb[k]))


@pytest.mark.parametrize("graph", [0, 1])
def test_rail_fp64_matches_oracle(lib, graph):
    from openradioss_b200.ecycle import ECycle
    from oracle.oracle import Oracle
    d = decks.hat_rail()
    g = ECycle(d, precision=abi.OR_PREC_FP64, lib=lib, graph=graph)
    o = Oracle(d, nthreads=8)
    g.step(150)
    o.step(150)
    # linked nodes move together (x, y linked; z held by the BCS)
    left = d["parts"][0]["rlinks"][0]["nodes"]
    v = g.get_nodes()["v"][left]
    assert np.all(v == v[0])
    compare(g, o, FP64_TOL, FP64_PLASTIC_IP_TOL)
    assert (o.shell_state(0)["pla"] > 0).mean() > 0.5          # the plastic branch is exercised
    # the link released between steps, as by an engine deck without the /VEL card
    g.set_rlink(0, 0, 0)
    o.set_rlink(0, 0, 0)
    g.step(150)
    o.step(150)
    compare(g, o, FP64_TOL, FP64_PLASTIC_IP_TOL)
    v = g.get_nodes()["v"][left]
    assert not np.all(v[:, 0] == v[0, 0])
    g.close()


def test_rail_split_matches_fp64_oracle(lib):
    from openradioss_b200.ecycle import ECycle
    from oracle.oracle import Oracle
    d = decks.hat_rail()
    g = ECycle(d, precision=abi.OR_PREC_SPLIT, lib=lib)
    o = Oracle(d, nthreads=8)
    g.step(100)
    o.step(100)
    a, b = g.get_nodes(), o.get_nodes()
    assert rel(a["d"], b["d"]) < SPLIT_TOL, rel(a["d"], b["d"])
    g.close()


def test_rail_options_outside_the_adjoint_and_domain_decomposition(lib):
    from openradioss_b200.ecycle import ECycle, ECycleError
    d = decks.hat_rail(length=0.05, kink=(0.02, 0.03))
    g = ECycle(d, precision=abi.OR_PREC_FP64, lib=lib)
    with pytest.raises(ECycleError) as e:
        g.adjoint(10, node=0, comp=0)
    assert e.value.code == abi.OR_E_UNSUPPORTED
    one = np.zeros(1, np.int32)
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    with pytest.raises(ECycleError) as e:
        g._call("set_halo", 0, 1, ip(one), ip(one), ip(one + 1), 1)
    assert e.value.code == abi.OR_E_UNSUPPORTED
    g.close()
