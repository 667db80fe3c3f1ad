"""Known answers for the shell formulations Ishell 1 to 4 and one-point shells
in the CPU oracle (the engine's IHBE 1, 0, 2, 4; cdefo3.F, chvis3.F,
chsti3.F, mhvis3.F, cfint3.F).

* A uniform membrane stretch has no hourglass and no warping: every
  formulation gives the stresses of sigeps01c.F.
* On a mesh of squares with exactly representable coordinates the CHVIS3 shape
  vectors are the plain +-1 vectors (VHX = VHY = 0), so Ishell 2 (IHBE 0) and
  Ishell 1 give the same bits.
* A pure membrane or bending hourglass velocity on one square: the elastic
  hourglass state after one cycle is the closed form of each routine
  (CHVIS3 and CHSTI3 with their own coefficients, MHVIS3 for one point).
* CHSTI3 bounds the membrane hourglass force by SIGY THK0 sqrt(A) hm / 2, with
  SIGY the mean yield stress of the integration points (sigeps02c.F:186):
  with a perfectly plastic law SIGY = A and the bound is reached.
"""
import math

import numpy as np
import pytest

from openradioss_b200 import decks
from oracle.oracle import Oracle

H = 1e-3
E, NU, RHO = 70e9, 0.33, 2700.0


def one_square(ishell, npt, v, vr=None, dt=1e-7, thk=1e-3, mat=None, hm=0.01, hf=0.01, hr=0.01, dn=0.0):
    x, conn, _ = decks.quad_plate(1, H)
    p = decks.new_part(x)
    mat = mat or decks.material(decks.LAW_ELASTIC, RHO, E, NU)
    decks.add_shell(p, conn, mat, decks.shell_prop(thk, npt=npt, ishell=ishell, hm=hm, hf=hf, hr=hr, dn=dn))
    p["v"] = v(x)
    if vr is not None:
        p["vr"] = vr(x)
    o = Oracle(decks.deck([p]))
    o.times[0].dt2 = dt
    return o


@pytest.mark.parametrize("npt", [1, 3, 5])
@pytest.mark.parametrize("ishell", [1, 2, 3, 4])
def test_membrane_stretch_is_formulation_independent(ishell, npt):
    edot, dt = 100.0, 1e-7
    o = one_square(ishell, npt, lambda x: np.stack([edot * x[:, 0], 0 * x[:, 0], 0 * x[:, 0]], 1), dt=dt)
    o.step(1)
    s = o.shell_state(0)
    mat = decks.material(decks.LAW_ELASTIC, RHO, E, NU)
    np.testing.assert_allclose(s["sig"][:, 0, 0], mat["a11"] * edot * dt, rtol=1e-12)
    np.testing.assert_allclose(s["sig"][:, 1, 0], mat["a12"] * edot * dt, rtol=1e-12)
    assert np.abs(s["hourg"]).max() < 1e-20 * mat["a11"]


@pytest.mark.parametrize("npt", [1, 5])
def test_ishell2_equals_ishell1_on_squares(npt):
    """One cycle from a seeded random velocity field: on squares with exact
    coordinates the forces of Ishell 1 and 2 agree to the bit; on a jittered mesh
    they differ, except with one point, where the starter turns Ishell 2 into 1
    (hm_read_prop01.F:246-250)."""
    def run(ishell, jitter):
        d = decks.c2_shell_plate(n=4, size=2.0 ** -7, npt=npt, pressure=6e6, ishell=ishell, jitter=jitter)
        p = d["parts"][0]
        rng = np.random.default_rng(5)
        p["v"] = rng.uniform(-1, 1, p["x"].shape)
        p["vr"] = rng.uniform(-100, 100, p["x"].shape)
        o = Oracle(d)
        o.times[0].dt2 = 1e-8
        o.step(1)
        return o.get_nodes(), o.shell_state(0)
    (na, sa), (nb, sb) = run(1, 0.0), run(2, 0.0)
    for k in ("v", "vr"):
        assert np.array_equal(na[k], nb[k]), k
    for k in ("sig", "hourg"):
        assert np.array_equal(sa[k], sb[k]), k
    (na, sa), (nb, sb) = run(1, 0.05), run(2, 0.05)
    assert np.array_equal(sa["hourg"], sb["hourg"]) == (npt == 1)


def hourglass_velocity(kind, w=1.0):
    """x, y, z hourglass pattern (+ - + -) over the corners of the square."""
    def f(x):
        s = np.where((x[:, 0] > 0) == (x[:, 1] > 0), 1.0, -1.0)   # corners 1, 3: +1; 2, 4: -1
        v = np.zeros_like(x)
        v[:, kind] = w * s
        return v
    return f


@pytest.mark.parametrize("ishell,npt", [(1, 5), (2, 5), (3, 5), (4, 5), (1, 1), (3, 1), (4, 1)])
def test_membrane_hourglass_state(ishell, npt):
    """HOUR1 after one cycle = HG1 * (elastic coefficient): 4 v hm YM THK0 DT1 / 8
    for CHVIS3 (A7 TD, HELAS = 1/2) and MHVIS3 (H1 FAC), and 4 v hm YM THK0 DT1 / 8
    for CHSTI3 (YM THK0 DT1 / 8, chsti3.F:136); IHBE 2 takes velocities relative to
    node 1 (cdefo3.F:140-150), which leaves HG1 unchanged."""
    w, dt, thk, hm = 0.3, 1e-7, 1e-3, 0.05
    o = one_square(ishell, npt, hourglass_velocity(0, w), dt=dt, thk=thk, hm=hm)
    o.step(1)
    got = o.shell_state(0)["hourg"][0, 0]
    want = 4 * w * hm * E * thk * dt / 8.0
    np.testing.assert_allclose(got, want, rtol=1e-12)


@pytest.mark.parametrize("ishell,npt", [(1, 5), (3, 5), (1, 1), (4, 1)])
def test_bending_hourglass_state(ishell, npt):
    """HOUR3 after one cycle: CHVIS3 hf YM/8 SHF/(3(1+nu)) THK0^3 DT1/(B1+B2) (chvis3.F:153-178),
    CHSTI3 the same with YM THK0 DT1 / 8 (chsti3.F:136-139), MHVIS3 hf YM THK0 DT1 / 8
    (mhvis3.F:153-158) -- each times HG = 4 w."""
    w, dt, thk, hf = 0.2, 1e-7, 1e-3, 0.04
    o = one_square(ishell, npt, hourglass_velocity(2, w), dt=dt, thk=thk, hf=hf)
    o.step(1)
    got = o.shell_state(0)["hourg"][2, 0]
    shf = 5.0 / 6.0
    b12 = H ** 2                    # B1 + B2 of a square of side H: PX, PY = +-H/2
    if npt == 1:
        want = 4 * w * hf * E * thk * dt / 8.0
    else:
        want = 4 * w * hf * E / 8.0 * shf / (3 * (1 + NU)) * thk ** 3 * dt / b12
    np.testing.assert_allclose(got, want, rtol=1e-10)


def test_one_point_v_shape_damping_moves_forces_not_state():
    """MHVIS3's V-shape term (Dn) acts on the forces only: the same state, other
    nodal velocities after one more cycle."""
    f = lambda x: np.stack([0 * x[:, 0], 0 * x[:, 0], np.where(x[:, 1] > 0, -0.2, 0.2)], 1)
    a = one_square(1, 1, f, dn=0.0)
    b = one_square(1, 1, f, dn=0.05)
    for o in (a, b):
        o.step(2)
    assert np.array_equal(a.shell_state(0)["hourg"], b.shell_state(0)["hourg"])
    assert not np.array_equal(a.get_nodes()["v"], b.get_nodes()["v"])


@pytest.mark.parametrize("kind", [0, 2])
def test_chsti3_bounds_the_hourglass_force_by_the_yield_stress(kind):
    """A fast hourglass velocity on one square of a perfectly plastic LAW2
    (SIGY = A): the elastic increment exceeds the bound in the first cycle, so
    HOUR1 = SIGY THK0 sqrt(AREA) hm / 2 (membrane) and HOUR3 = SIGY THK0^2 hf / 4
    (bending), chsti3.F:247-280."""
    ca, thk, hm, hf = 2e6, 1e-3, 0.1, 0.1
    mat = decks.material(decks.LAW_JOHNSON_COOK, RHO, E, NU, jc_a=ca, jc_b=0.0, jc_n=1.0)
    o = one_square(3, 5, hourglass_velocity(kind, 5.0), mat=mat, thk=thk, hm=hm, hf=hf)
    o.step(1)
    h = o.shell_state(0)["hourg"][:, 0]
    sigy = sum([ca / 5.0] * 5)                      # SIGY = sum of YLD / NPTT
    if kind == 0:
        np.testing.assert_allclose(h[0], 0.5 * sigy * thk * H * hm, rtol=1e-12)
    else:
        np.testing.assert_allclose(h[2], 0.25 * sigy * thk * thk * hf, rtol=1e-12)
    # LAW1 leaves SIGY at EP30: no bound, the elastic increment
    o = one_square(3, 5, hourglass_velocity(kind, 5.0), thk=thk, hm=hm, hf=hf)
    o.step(1)
    h = o.shell_state(0)["hourg"][:, 0]
    if kind == 0:
        np.testing.assert_allclose(h[0], 4 * 5.0 * hm * E * thk * 1e-7 / 8.0, rtol=1e-12)
