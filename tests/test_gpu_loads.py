"""Parity of the sm_100a path with the CPU oracle on decks with /CLOAD and
/PLOAD loads driven by /FUNCT time functions, and with skewed /BCS
(force.F90, tools/curve/finter.F, bcs1.F BCS1V):

* a jittered shell plate with a force ramp and a moment at two nodes (one in a
  skew frame), a pressure history on quadrangle and triangle segments, and one
  edge held along the z' axis of a skew frame;
* a hexa block with a pressure on its top face and its base held in a skew
  frame.

Tolerances as in test_gpu_parity.py: FP64 1e-10 normwise on nodal
displacements and velocities, time and energies (external work included);
split form 1e-5 on displacements against the FP64 oracle.
"""
import numpy as np
import pytest

from openradioss_b200 import abi, decks

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
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


def skew_axes(angle, axis=0):
    c, s = np.cos(angle), np.sin(angle)
    R = np.eye(3)
    i, j = [(1, 2), (2, 0), (0, 1)][axis]
    R[i, i], R[i, j], R[j, i], R[j, j] = c, -s, s, c
    return R.T.reshape(9)                   # rows: x', y', z'


def shell_deck():
    n = 20
    x, conn, edge = decks.quad_plate(n, 0.02, jitter=0.05, seed=3)
    p = decks.new_part(x)
    decks.add_shell(p, conn, decks.aluminium_jc(), decks.shell_prop(1e-3, npt=5))
    left = np.nonzero(np.isclose(x[:, 0], 0.0))[0]
    others = np.nonzero(edge & ~np.isclose(x[:, 0], 0.0))[0]
    p["icodt"][others] = 1
    p["icodt"][left] = 3                      # y', z' held in a frame rotated about x
    p["icodr"][left] = 4
    p["iskew"] = -np.ones(x.shape[0], np.int32)
    p["iskew"][left] = 0
    centre = int(np.argmin(np.linalg.norm(x - [0.01, 0.01, 0.0], axis=1)))
    quarter = int(np.argmin(np.linalg.norm(x - [0.015, 0.005, 0.0], axis=1)))
    p["cloads"] = [dict(nodes=np.array([centre]), dir=3, func=0, ascale_x=1.0, fscale=-40.0),
                   dict(nodes=np.array([quarter]), dir=4, skew=1, func=1, ascale_x=2.0, fscale=0.02)]
    half = conn[: conn.shape[0] // 2]
    tri = conn[conn.shape[0] // 2: conn.shape[0] // 2 + 20].copy()
    tri[:, 3] = -1                            # three-node segments
    p["ploads"] = [dict(seg=half, func=1, ascale_x=1.0, fscale=2e5),
                   dict(seg=tri, func=0, ascale_x=0.5, fscale=-1e5)]
    d = decks.deck([p], name="shell_loads")
    d["functions"] = [dict(x=[0.0, 5e-6, 2e-5], y=[0.0, 1.0, 0.3]),
                      dict(x=[0.0, 1e-5, 2e-5, 3e-5], y=[0.2, 1.0, -0.5, 0.4])]
    d["skews"] = [skew_axes(0.4, axis=0), skew_axes(0.7, axis=2)]
    return d


def hex_deck():
    x, conn = decks.hex_block(4, 4, 8, 1e-3)
    p = decks.new_part(x)
    decks.add_hex(p, conn, decks.steel_jc(), decks.solid_prop())
    base = np.nonzero(np.isclose(x[:, 2], 0.0))[0]
    p["icodt"][base] = 5                      # x', z' held
    p["iskew"] = -np.ones(x.shape[0], np.int32)
    p["iskew"][base] = 0
    top = conn[np.isclose(x[conn[:, 4], 2], 8e-3)][:, 4:8]
    p["ploads"] = [dict(seg=top, func=0, ascale_x=1.0, fscale=-1e8)]
    corner = int(np.argmin(np.linalg.norm(x - [4e-3, 4e-3, 8e-3], axis=1)))
    p["cloads"] = [dict(nodes=np.array([corner]), dir=1, skew=0, func=0, fscale=20.0)]
    d = decks.deck([p], name="hex_loads")
    d["functions"] = [dict(x=[0.0, 2e-6, 1e-5], y=[0.0, 1.0, 1.0])]
    d["skews"] = [skew_axes(0.5, axis=2)]
    return d


def compare(g, o, tol):
    a, b = g.get_nodes(), o.get_nodes()
    for k in ("d", "v", "vr"):
        if np.abs(b[k]).max() > 0:
            assert rel(a[k], b[k]) < tol, (k, rel(a[k], b[k]))
    ta, tb = g.time(), o.time()
    assert ta["ncycle"] == tb["ncycle"]
    assert abs(ta["tt"] - tb["tt"]) <= tol * tb["tt"]
    ea, eb = g.energies(), o.energies()
    for k in ("internal", "kinetic", "kinetic_rot", "hourglass", "external_work"):
        assert abs(ea[k] - eb[k]) <= tol * max(abs(eb[k]), 1e-300), (k, ea[k], eb[k])


@pytest.mark.parametrize("make", [shell_deck, hex_deck], ids=["shell", "hex"])
def test_loads_fp64_match_oracle(lib, make):
    from openradioss_b200.ecycle import ECycle
    from oracle.oracle import Oracle
    d = make()
    g = ECycle(d, precision=abi.OR_PREC_FP64, lib=lib)
    o = Oracle(d, nthreads=8)
    for n in (7, 60, 93):                     # several step calls: graph replays of partial batches
        g.step(n)
        o.step(n)
    assert o.energies()["external_work"] != 0.0
    compare(g, o, FP64_TOL)
    # held directions of the skewed nodes stay at rest
    p = d["parts"][0]
    v = g.get_nodes()["v"]
    zp = np.asarray(d["skews"][0])[6:9]
    held = np.nonzero(p["iskew"] >= 0)[0]
    assert np.abs(v[held] @ zp).max() <= 1e-12 * np.abs(v).max()
    g.close()


@pytest.mark.parametrize("make", [shell_deck, hex_deck], ids=["shell", "hex"])
def test_loads_split_match_fp64_oracle(lib, make):
    from openradioss_b200.ecycle import ECycle
    from oracle.oracle import Oracle
    d = make()
    g = ECycle(d, precision=abi.OR_PREC_SPLIT, lib=lib)
    o = Oracle(d, nthreads=8)
    g.step(120)
    o.step(120)
    a, b = g.get_nodes(), o.get_nodes()
    assert rel(a["d"], b["d"]) < SPLIT_TOL, rel(a["d"], b["d"])
    g.close()
