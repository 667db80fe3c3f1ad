"""The FP64 reference gradient (adjoint_reference.py) against central finite
differences of the oracle, on the CPU.

Deck: the adjoint plate at 6x6 (per-element Johnson-Cook A and thickness
drawn as in the C5 workload), linear hardening so that a 1e-7 relative step
stays inside the linear region, DTMX below every element time step so that
the dt sequence does not depend on the parameters.  The thickness derivative
includes the nodal-mass chain of the deck builder's lumping, as for the GPU
adjoint.
"""
import numpy as np
import pytest

from openradioss_b200 import adjoint, decks

import adjoint_reference as ref

DTMX = 1.4e-7


def plate(n, A, T, pressure, ncycles):
    d = decks.c2_shell_plate(n=n, size=n * 1e-3, pressure=pressure, ncycles=ncycles, jc_a=A, thke=T)
    d["parts"][0]["shell"][0]["mat"]["jc_n"] = 1.0
    d["dtmx"] = DTMX
    return d


def base(n, seed=1):
    g = decks.c5_adjoint_plate(n=n, seed=seed)["parts"][0]["shell"][0]
    return np.array(g["jc_a"]), np.array(g["thke"])


def oracle_J(deck, ncycles, node, wd, wp):
    from oracle.oracle import Oracle
    from openradioss_b200 import abi
    o = Oracle(deck, precision=abi.OR_PREC_FP64)
    w0 = o.energies()["plastic_work"]
    o.step(ncycles)
    J = wd * o.get_nodes()["d"][node, 2] + wp * (o.energies()["plastic_work"] - w0)
    o.close()
    return J


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    return ref.build_host_lib(tmp_path_factory.mktemp("adjref"))


@pytest.mark.parametrize("wd,wp", [(1.0, 0.0), (0.0, 1.0)])
def test_reference_gradient_matches_central_differences(lib, wd, wp):
    n, N, p, STEP = 6, 60, 3e7, 1e-7
    A0, T0 = base(n)
    d0 = plate(n, A0, T0, p, N)
    node = adjoint.centre_node(d0)
    res = ref.reference_gradient(d0, N, node, 2, wd, wp, lib)
    assert res["J"] == oracle_J(d0, N, node, wd, wp)
    if wp:
        assert res["J"] > 0.0 and np.abs(res["dA"][0]).max() > 0.0
    gA, gT = res["dA"][0], adjoint.thickness_gradient(d0, res)[0]
    rng = np.random.default_rng(7)
    for name in ("A", "thk", "both"):
        uA = rng.choice([-1.0, 1.0], A0.size) if name in ("A", "both") else 0.0 * A0
        uT = rng.choice([-1.0, 1.0], T0.size) if name in ("thk", "both") else 0.0 * T0
        Jp = oracle_J(plate(n, A0 * (1 + STEP * uA), T0 * (1 + STEP * uT), p, N), N, node, wd, wp)
        Jm = oracle_J(plate(n, A0 * (1 - STEP * uA), T0 * (1 - STEP * uT), p, N), N, node, wd, wp)
        fd = (Jp - Jm) / (2 * STEP)
        ad = float(np.dot(gA, A0 * uA) + np.dot(gT, T0 * uT))
        assert abs(fd - ad) <= 1e-4 * abs(ad), (name, fd, ad)
