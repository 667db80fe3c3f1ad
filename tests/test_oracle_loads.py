"""Known answers for the oracle's loads and skewed boundary conditions (the
restatement of force.F90, tools/curve/finter.F and bcs1.F BCS1V):

* a /CLOAD ramp on a free plate: the total momentum after N cycles is the sum of
  the cycles' DT12 * F(TT) with F from FINTER (linear extrapolation past the
  last point included);
* a /PLOAD on a free flat plate: momentum grows as p * area * normal;
* a skewed /BCS: the velocity of a node held along the skew z' axis has no
  z' component, whatever load pushes it;
* the external work of a constant concentrated load is the sum over cycles of F
  times the node velocity at the cycle's start times the cycle's DT2
  (WFEXC * DT2, resol.F:6238).
"""
import numpy as np
import pytest

from openradioss_b200 import decks


def free_plate(n=4, size=0.02):
    x, conn, _ = decks.quad_plate(n, size)
    p = decks.new_part(x)
    decks.add_shell(p, conn, decks.steel_elastic(), decks.shell_prop(1e-3, npt=3, ithk=0))
    return p, x, conn


def finter_ref(x, y, t):
    """FINTER by hand: piecewise linear, linear extrapolation at both ends."""
    x, y = np.asarray(x), np.asarray(y)
    if x.size == 1:
        return y[0]
    i = int(np.clip(np.searchsorted(x, t), 1, x.size - 1))
    return y[i - 1] + (t - x[i - 1]) * (y[i] - y[i - 1]) / (x[i] - x[i - 1])


def run_steps(o, n):
    hist = []
    for _ in range(n):
        t0 = o.time()["tt"]
        o.step(1)
        hist.append((t0, o.time()["dt12"]))
    return hist


def test_cload_ramp_momentum():
    from oracle.oracle import Oracle
    p, x, conn = free_plate()
    fx, fy = [0.0, 2e-6, 3e-6], [0.0, 50.0, 60.0]        # 3 points; run beyond the last
    p["cloads"] = [dict(nodes=np.array([0, 7]), dir=2, func=0, ascale_x=1.0, fscale=2.0)]
    d = decks.deck([p])
    d["functions"] = [dict(x=fx, y=fy)]
    o = Oracle(d)
    hist = run_steps(o, 60)
    mom = (o.get_nodes()["v"][:, 1] * p["ms"]).sum()
    want = sum(dt12 * 2.0 * 2.0 * finter_ref(fx, fy, tt) for tt, dt12 in hist)
    assert o.time()["tt"] > fx[-1]                        # extrapolation reached
    assert mom == pytest.approx(want, rel=1e-12)


def test_pload_total_force():
    from oracle.oracle import Oracle
    p, x, conn = free_plate()
    p["ploads"] = [dict(seg=conn, func=0, ascale_x=1.0, fscale=-3e5)]
    d = decks.deck([p])
    d["functions"] = [dict(x=[0.0], y=[1.0])]             # constant
    o = Oracle(d)
    hist = run_steps(o, 20)
    mom = (o.get_nodes()["v"] * p["ms"][:, None]).sum(axis=0)
    area = 0.02 * 0.02
    want = sum(dt12 for _, dt12 in hist) * (-3e5) * area   # along +z: (x3-x1) x (x4-x2) = +z
    assert mom[2] == pytest.approx(want, rel=1e-9)
    assert abs(mom[0]) < 1e-12 * abs(want) and abs(mom[1]) < 1e-12 * abs(want)


def test_skewed_bcs_removes_the_held_direction():
    from oracle.oracle import Oracle
    p, x, conn = free_plate()
    c, s = np.cos(0.3), np.sin(0.3)
    axes = [1.0, 0.0, 0.0, 0.0, c, s, 0.0, -s, c]         # x', y', z' = rotation about x
    p["iskew"] = -np.ones(x.shape[0], np.int32)
    held = np.arange(x.shape[0])
    p["iskew"][held] = 0
    p["icodt"][held] = 1                                  # z' held
    p["cloads"] = [dict(nodes=np.array([3]), dir=3, func=0, fscale=100.0)]
    d = decks.deck([p])
    d["functions"] = [dict(x=[0.0], y=[1.0])]
    d["skews"] = [axes]
    o = Oracle(d)
    o.step(30)
    v = o.get_nodes()["v"]
    zp = np.array(axes[6:9])
    assert np.abs(v @ zp).max() < 1e-12 * np.abs(v).max()
    assert np.abs(v[3]).max() > 0                         # the load moves it in the y' direction


def test_external_work_of_constant_cload():
    from oracle.oracle import Oracle
    p, x, conn = free_plate(n=1, size=0.01)
    p["cloads"] = [dict(nodes=np.arange(4), dir=1, func=0, fscale=10.0)]
    d = decks.deck([p])
    d["functions"] = [dict(x=[0.0], y=[1.0])]
    o = Oracle(d)
    want = 0.0
    for _ in range(40):
        v0 = o.get_nodes()["v"][:, 0].copy()      # velocity at the cycle's start
        o.step(1)
        want += 10.0 * v0.sum() * o.time()["dt2"]  # WFEXC = F.v, times the cycle's DT2
    assert want > 0
    assert o.energies()["external_work"] == pytest.approx(want, rel=1e-12)
