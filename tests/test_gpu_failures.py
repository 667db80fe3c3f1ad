"""Failure paths of the handle, each made on the host or by a deck the device
checks itself, never by a GPU fault.

* OR_E_DTMIN: DTMIN above every element time step (MQVISCB / CDT3 compare each
  element's step with DTMIN1; here that stops the run and names the element);
* OR_E_NAN: a non-finite velocity set between steps; the node pass finds the
  non-finite acceleration it produces and names the node;
* OR_E_TIMEOUT: the host's bounded wait given a limit far below the run's
  length; the cycles finish on the GPU, the handle is then destroyed cleanly;
  and the persistent cycle's grid barrier, with one CTA held back from the first
  barrier by the OR_ECYCLE_TEST_STALL_CTA hook: the others give up after about a
  second, set the abort flag and return, the step reports OR_E_TIMEOUT, and the
  handle runs again after a reset;
* upload rejections: node numbers outside the part in IXS / IXC, non-positive
  shell thickness, non-finite coordinates or velocities.
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


@pytest.mark.parametrize("precision", [abi.OR_PREC_FP64, abi.OR_PREC_SPLIT])
def test_dtmin_solid_reports_element(lib, precision):
    from openradioss_b200.ecycle import ECycle, ECycleError
    d = decks.c1_hex_block(nx=3, ny=3, nz=6)
    g = ECycle(d, precision=precision, dtmin_solid=1.0)     # every element's dt is ~1e-7 s
    with pytest.raises(ECycleError) as ei:
        g.step(4)
    code, idx = g.error_info()
    assert ei.value.code == code == abi.OR_E_DTMIN
    assert 0 <= idx < 54


@pytest.mark.parametrize("precision", [abi.OR_PREC_FP64, abi.OR_PREC_SPLIT])
def test_dtmin_shell_reports_element(lib, precision):
    from openradioss_b200.ecycle import ECycle, ECycleError
    d = decks.c2_shell_plate(n=8, size=8e-3)
    g = ECycle(d, precision=precision, dtmin_shell=1.0)
    with pytest.raises(ECycleError) as ei:
        g.step(4)
    code, idx = g.error_info()
    assert ei.value.code == code == abi.OR_E_DTMIN
    assert 0 <= idx < 64
    # a DTMIN below every element's step leaves the same deck running
    ok = ECycle(d, precision=precision, dtmin_shell=1e-12)
    ok.step(4)


@pytest.mark.parametrize("precision", [abi.OR_PREC_FP64, abi.OR_PREC_SPLIT])
def test_nan_velocity_reports_node(lib, precision):
    from openradioss_b200.ecycle import ECycle, ECycleError
    d = decks.c1_hex_block(nx=3, ny=3, nz=6)
    g = ECycle(d, precision=precision)
    g.step(5)
    v = g.get_nodes()["v"]
    bad = 37
    v[bad, 1] = np.nan
    g.set_nodes(0, v=v)
    with pytest.raises(ECycleError) as ei:
        g.step(2)
    code, idx = g.error_info()
    assert ei.value.code == code == abi.OR_E_NAN
    # the node named is one of the nodes the non-finite velocity reached: the
    # corners of the hexas around node `bad`
    conn = d["parts"][0]["hex"][0]["ixs"][:, 1:9] - 1
    touched = np.unique(conn[(conn == bad).any(axis=1)])
    assert idx in touched


def test_bounded_wait_expires_then_handle_closes(lib):
    import torch
    from openradioss_b200.ecycle import ECycle, ECycleError
    d = decks.c2_shell_plate(n=64, size=0.064)
    g = ECycle(d, precision=abi.OR_PREC_SPLIT)
    g.step(64)                                  # graph captured, context warm
    old = os.environ.get("OR_ECYCLE_TIMEOUT_S")
    os.environ["OR_ECYCLE_TIMEOUT_S"] = "1e-6"
    try:
        with pytest.raises(ECycleError) as ei:
            g.step(4000)                        # tens of ms of cycles
        assert ei.value.code == abi.OR_E_TIMEOUT
    finally:
        if old is None:
            del os.environ["OR_ECYCLE_TIMEOUT_S"]
        else:
            os.environ["OR_ECYCLE_TIMEOUT_S"] = old
    torch.cuda.synchronize()                    # the cycles finish normally
    g.close()
    # the device is usable afterwards
    h = ECycle(d, precision=abi.OR_PREC_SPLIT)
    h.step(64)
    assert np.isfinite(h.get_nodes()["d"]).all()


def test_persistent_barrier_wait_expires(lib, monkeypatch):
    import torch
    from openradioss_b200.ecycle import ECycle, ECycleError
    d = decks.c2_shell_plate(n=40, size=0.04)
    monkeypatch.setenv("OR_ECYCLE_TEST_STALL_CTA", "3")
    g = ECycle(d, precision=abi.OR_PREC_SPLIT)
    monkeypatch.delenv("OR_ECYCLE_TEST_STALL_CTA")
    on, ctas, _ = g.persistent_info()
    assert on and ctas > 3
    with pytest.raises(ECycleError) as ei:
        g.step(8)
    assert ei.value.code == abi.OR_E_TIMEOUT
    code, idx = g.error_info()
    assert code == abi.OR_E_TIMEOUT and 0 <= idx < ctas
    torch.cuda.synchronize()                    # the kernel returned; the context is usable
    g.close()
    h = ECycle(d, precision=abi.OR_PREC_SPLIT)
    r = ECycle(d, precision=abi.OR_PREC_SPLIT, persistent=-1)
    h.step(8)
    r.step(8)
    assert h.persistent_info()[0]
    assert np.abs(h.get_nodes()["d"] - r.get_nodes()["d"]).max() <= 1e-5 * np.abs(r.get_nodes()["d"]).max()


def _expect_arg_error(deck):
    from openradioss_b200.ecycle import ECycle, ECycleError
    with pytest.raises(ECycleError) as ei:
        ECycle(deck)
    assert ei.value.code == abi.OR_E_ARG


@pytest.mark.parametrize("node", [0, 10 ** 6])
def test_upload_rejects_ixs_out_of_range(lib, node):
    d = decks.c1_hex_block(nx=2, ny=2, nz=2)
    d["parts"][0]["hex"][0]["ixs"][3, 4] = node          # 1-based: 0 and > numnod are outside
    _expect_arg_error(d)


@pytest.mark.parametrize("node", [0, 10 ** 6])
def test_upload_rejects_ixc_out_of_range(lib, node):
    d = decks.c2_shell_plate(n=4, size=4e-3)
    d["parts"][0]["shell"][0]["ixc"][2, 3] = node
    _expect_arg_error(d)


@pytest.mark.parametrize("thk", [0.0, -1e-3])
def test_upload_rejects_non_positive_thickness(lib, thk):
    d = decks.c2_shell_plate(n=4, size=4e-3)
    g = d["parts"][0]["shell"][0]
    t = np.full(g["ixc"].shape[0], 1e-3)
    t[5] = thk
    g["thke"] = t
    _expect_arg_error(d)


@pytest.mark.parametrize("field", ["x", "v"])
def test_upload_rejects_non_finite_nodes(lib, field):
    d = decks.c1_hex_block(nx=2, ny=2, nz=2)
    d["parts"][0][field][4, 2] = np.inf if field == "x" else np.nan
    _expect_arg_error(d)
