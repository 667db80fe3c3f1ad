"""Restart through the C-ABI: a run of N cycles whose nodes, element state,
time state and cumulative energies are copied into a fresh handle
(or_ecycle_set_nodes, or_ecycle_set_hex_state, or_ecycle_set_shell_state,
or_ecycle_set_energy_sums), then M more cycles, must equal N + M cycles of one
handle: the nodes bitwise, the cumulative energies to their summation order.

Decks: the mixed hexa/shell mesh, and the crash rail with its rigid link and
loads added (/CLOAD ramp, /PLOAD), in both precision forms.
"""
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


def rail_with_loads():
    d = decks.hat_rail(length=0.15, kink=(0.05, 0.1))
    p = d["parts"][0]
    x = p["x"]
    far = np.nonzero(np.isclose(x[:, 0], x[:, 0].max()))[0]
    p["cloads"] = [dict(nodes=far[:3], dir=2, func=0, fscale=200.0)]
    conn = p["shell"][0]["ixc"][:, 1:5] - 1
    p["ploads"] = [dict(seg=conn[:40], func=0, fscale=-1e5)]
    d["functions"] = [dict(x=[0.0, 1e-4], y=[0.0, 1.0])]
    return d


@pytest.mark.parametrize("precision", [abi.OR_PREC_FP64, abi.OR_PREC_SPLIT], ids=["fp64", "split"])
@pytest.mark.parametrize("make", [lambda: decks.c4_mixed_mesh(nx=6, ny=6, nz=12), rail_with_loads],
                         ids=["mixed", "rail"])
def test_restart_equals_continuous_run(lib, make, precision):
    from openradioss_b200.ecycle import ECycle
    d = make()
    n, m = 70, 90
    one = ECycle(d, precision=precision, lib=lib)
    one.step(n + m)
    first = ECycle(d, precision=precision, lib=lib)
    first.step(n)
    second = ECycle(d, precision=precision, lib=lib)
    second.restart_from(first)
    second.step(m)
    a, b = second.get_nodes(), one.get_nodes()
    for k in ("x", "d", "v", "vr"):
        assert np.array_equal(a[k], b[k]), k
    ta, tb = second.time(), one.time()
    assert ta["tt"] == tb["tt"] and ta["dt2"] == tb["dt2"]
    ea, eb = second.energies(), one.energies()
    for k in ("internal", "kinetic", "kinetic_rot"):
        assert ea[k] == eb[k], k
    for k in ("hourglass", "plastic_work", "external_work"):
        assert ea[k] == pytest.approx(eb[k], rel=1e-13, abs=0), k
    for gi in range(len(one.shell_groups)):
        sa, sb = second.shell_state(gi), one.shell_state(gi)
        for k in sa:
            assert np.array_equal(sa[k], sb[k]), k
    for h in (one, first, second):
        h.close()
