"""Adjoint of the shell cycle (or_ecycle_adjoint) against central finite
differences of the forward cycle, on the GPU.

Workload: the adjoint plate (per-element Johnson-Cook A ~ U(300, 400) MPa and
thickness ~ U(0.9, 1.1) mm, simply supported, uniform pressure), with DTMX
below every element time step so that the dt sequence is the same constant in
every run: the adjoint holds dt fixed, and with DTMX binding the forward does
too, so the finite differences measure the same derivative.

Responses: the z displacement of the centre node at the end, and the plastic
work of the run.  Parameters: the elements' A and thickness (the nodal masses
follow the thickness through the deck builder's lumping; the adjoint returns
dJ/dMS and dJ/dIN and openradioss_b200.adjoint adds that chain).  Bar: 1e-4
relative, central differences along random directions.

The finite-difference step must stay inside the region where the response is
linear, and that region depends on the hardening law:
- elastic (LAW1): J is smooth; a 1e-6 relative step agrees to ~1e-9.
- LAW2 with linear hardening (n = 1): a 1e-6 step straddles yield-onset kinks
  of a few integration points (up to 5e-4 off); 1e-7 agrees to better than 1e-6.
- LAW2 with the aluminium's n = 0.36: the hardening slope B n eps_p^(n-1) is
  singular at first yield, where the first plastic increment can be smaller
  than the change a 1e-6 step in A causes (A/E * 1e-6 ~ 5e-9), so J is far
  from linear at that scale (1e-6 is off by O(1)).  On the 32x32 plate the
  differences converge to the adjoint as the step shrinks: 1e-8 agrees within
  1e-4.  On the full 200x200 plate some point yields with a far smaller first
  increment, and the plastic work's derivative with respect to A, which scales
  like eps_p^(n-1) there, is too large for any difference quotient to follow
  (it grows as the step shrinks); the displacement response is still checked.

The torch.autograd.Function below exists only for torch.autograd.gradcheck.
"""
import numpy as np
import pytest

from openradioss_b200 import abi, adjoint, decks

pytestmark = pytest.mark.gpu

DTMX = 1.4e-7
FD_REL = 1e-4


def need_gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openradioss_b200 import build
    build.build()


def plate(n, A, thk, pressure, ncycles, law=decks.LAW_JOHNSON_COOK, jc_n=0.36):
    d = decks.c2_shell_plate(n=n, size=n * 1e-3, pressure=pressure, ncycles=ncycles, jc_a=A, thke=thk, law=law)
    d["parts"][0]["shell"][0]["mat"]["jc_n"] = jc_n
    d["dtmx"] = DTMX
    return d


def base_params(n, seed=1):
    d = decks.c5_adjoint_plate(n=n, seed=seed)
    g = d["parts"][0]["shell"][0]
    return np.array(g["jc_a"]), np.array(g["thke"])


def forward_J(deck, ncycles, node, w_disp, w_plastic):
    """J of a regular step() on the per-phase kernels, the adjoint's forward."""
    from openradioss_b200.ecycle import ECycle
    h = ECycle(deck, precision=abi.OR_PREC_FP64, persistent=-1)
    wp0 = h.energies()["plastic_work"]
    h.step(ncycles)
    J = w_disp * h.get_nodes()["d"][node, 2] + w_plastic * (h.energies()["plastic_work"] - wp0)
    t = h.time()
    h.close()
    return J, t


def adjoint_run(deck, ncycles, node, w_disp, w_plastic, checkpoint=50):
    from openradioss_b200.ecycle import ECycle
    h = ECycle(deck, precision=abi.OR_PREC_FP64)
    res = h.adjoint(ncycles, node=node, comp=2, w_disp=w_disp, w_plastic=w_plastic, checkpoint=checkpoint)
    res["time"] = h.time()
    res["nodes"] = h.get_nodes()
    res["energies"] = h.energies()
    h.close()
    return res


CASES = [  # label, law, hardening exponent, pressure, cycles, response, FD step, bar
    ("elastic", decks.LAW_ELASTIC, 1.0, 2e6, 300, "disp", 1e-6, 1e-6),
    ("linear-hardening", decks.LAW_JOHNSON_COOK, 1.0, 2e6, 300, "disp", 1e-7, FD_REL),
    ("linear-hardening", decks.LAW_JOHNSON_COOK, 1.0, 2e6, 300, "plastic", 1e-7, FD_REL),
    ("linear-hardening", decks.LAW_JOHNSON_COOK, 1.0, 1e7, 200, "disp", 1e-7, FD_REL),
    ("linear-hardening", decks.LAW_JOHNSON_COOK, 1.0, 1e7, 200, "plastic", 1e-7, FD_REL),
    ("jc-0.36", decks.LAW_JOHNSON_COOK, 0.36, 2e6, 300, "disp", 1e-8, FD_REL),
    ("jc-0.36", decks.LAW_JOHNSON_COOK, 0.36, 2e6, 300, "plastic", 1e-8, FD_REL),
    ("jc-0.36", decks.LAW_JOHNSON_COOK, 0.36, 1e7, 200, "disp", 1e-8, FD_REL),
    ("jc-0.36", decks.LAW_JOHNSON_COOK, 0.36, 1e7, 200, "plastic", 1e-8, FD_REL),
]


def directional_check(n, law, jcn, pressure, ncycles, wd, wpl, step, bar, directions):
    A0, T0 = base_params(n)
    d0 = plate(n, A0, T0, pressure, ncycles, law, jcn)
    node = adjoint.centre_node(d0)
    res = adjoint_run(d0, ncycles, node, wd, wpl)
    # dt held at DTMX in every cycle: tt = ncycles * DTMX
    assert abs(res["time"]["tt"] - ncycles * DTMX) <= 1e-12 * ncycles * DTMX
    J0, _ = forward_J(d0, ncycles, node, wd, wpl)
    assert res["J"] == J0                     # the adjoint's forward is the regular cycle
    gA = res["dA"][0]
    gT = adjoint.thickness_gradient(d0, res)[0]
    if law == decks.LAW_ELASTIC:
        assert not gA.any()
    rng = np.random.default_rng(11)
    out = {}
    for name in directions:
        uA = rng.choice([-1.0, 1.0], A0.size) if name in ("A", "both") else 0.0 * A0
        uT = rng.choice([-1.0, 1.0], T0.size) if name in ("thk", "both") else 0.0 * T0
        Jp, tp = forward_J(plate(n, A0 * (1 + step * uA), T0 * (1 + step * uT), pressure, ncycles, law, jcn),
                           ncycles, node, wd, wpl)
        Jm, tm = forward_J(plate(n, A0 * (1 - step * uA), T0 * (1 - step * uT), pressure, ncycles, law, jcn),
                           ncycles, node, wd, wpl)
        assert tp["tt"] == tm["tt"] == res["time"]["tt"]
        fd = (Jp - Jm) / (2 * step)
        ad = float(np.dot(gA, A0 * uA) + np.dot(gT, T0 * uT))
        out[name] = (fd, ad)
        assert abs(fd - ad) <= bar * abs(ad), (name, fd, ad)
    return res, out


@pytest.mark.parametrize("label,law,jcn,pressure,ncycles,resp,step,bar", CASES)
def test_adjoint_matches_central_differences(label, law, jcn, pressure, ncycles, resp, step, bar):
    need_gpu()
    wd, wpl = (1.0, 0.0) if resp == "disp" else (0.0, 1.0)
    dirs = ("thk",) if law == decks.LAW_ELASTIC else ("A", "thk", "both")
    res, _ = directional_check(32, law, jcn, pressure, ncycles, wd, wpl, step, bar, dirs)
    if resp == "plastic":
        assert res["J"] > 0.0


def test_adjoint_full_size_c5_linear_hardening():
    """The C5 workload's size (200x200 plate, 500 cycles, 2 MPa) with linear
    hardening: both responses together, along A, thickness and both."""
    need_gpu()
    res, out = directional_check(200, decks.LAW_JOHNSON_COOK, 1.0, 2e6, 500, 1.0, 1.0, 1e-7, FD_REL,
                                 ("A", "thk", "both"))
    assert res["J"] > 0.0


def test_adjoint_full_size_c5_displacement():
    """The C5 workload as specified (aluminium n = 0.36): the centre-node
    displacement response along the thickness direction.  (Along A the
    displacement's sensitivity, ~2e-8 m per unit relative change, is below the
    rounding noise of a difference quotient; the plastic work's sensitivity to A
    is unbounded for n < 1 at first-yield points, see the module docstring.)"""
    need_gpu()
    directional_check(200, decks.LAW_JOHNSON_COOK, 0.36, 2e6, 500, 1.0, 0.0, 1e-8, FD_REL, ("thk",))


@pytest.mark.parametrize("wd,wp", [(1.0, 0.0), (0.0, 1.0), (1.0, 0.5)])
def test_adjoint_matches_fp64_reference_gradient(tmp_path, wd, wp):
    """Every component of dJ/dA, dJ/dthk, dJ/dMS and dJ/dIN against the FP64
    reference gradient of tests/adjoint_reference.py (oracle forward, host
    reverse of the nodal update and the assembly, checked against central
    differences in test_adjoint_reference.py): 6x6 adjoint plate, 60 cycles,
    30 MPa (plastic), linear hardening, checkpoints every 16 cycles."""
    need_gpu()
    import adjoint_reference as ref
    lib = ref.build_host_lib(tmp_path)
    n, N, p = 6, 60, 3e7
    A0, T0 = base_params(n)
    d0 = plate(n, A0, T0, p, N, jc_n=1.0)
    node = adjoint.centre_node(d0)
    res = adjoint_run(d0, N, node, wd, wp, checkpoint=16)
    rf = ref.reference_gradient(d0, N, node, 2, wd, wp, lib)
    assert abs(res["J"] - rf["J"]) <= 1e-12 * abs(rf["J"]), (res["J"], rf["J"])
    for k in ("dA", "dthk", "dms", "din"):
        g, r = res[k][0], rf[k][0]
        scale = np.abs(r).max()
        assert scale > 0.0 or (k == "dA" and wp == 0.0 and not g.any()), k
        assert np.abs(g - r).max() <= 1e-9 * scale, (k, np.abs(g - r).max(), scale)


def with_frame_skew_cloads(d):
    """The plate with /SHFRA/V4 element frames (ISHFRAM 2), its x = xmin edge
    held in a skew frame tilted 25 degrees about y (x' and z' held, and the
    rotation about y'), a ramped point load at the centre along z, and one along
    the skew frame's y' at the middle of the skewed edge."""
    P = d["parts"][0]
    P["shell"][0]["prop"]["ishfram"] = 2
    c, s = np.cos(np.radians(25.0)), np.sin(np.radians(25.0))
    d["skews"] = [np.array([[c, 0.0, -s], [0.0, 1.0, 0.0], [s, 0.0, c]])]
    d["functions"] = [{"x": np.array([0.0, 2e-5, 1.0]), "y": np.array([0.0, 1.0, 1.0])}]
    x = P["x"]
    left = np.nonzero(x[:, 0] <= x[:, 0].min() + 1e-9)[0]
    P["icodt"][left] = 5
    P["icodr"][left] = 2
    P["iskew"] = -np.ones(x.shape[0], np.int32)
    P["iskew"][left] = 0
    mid = int(left[np.argmin(np.abs(x[left, 1] - 0.5 * (x[:, 1].min() + x[:, 1].max())))])
    P["cloads"] = [dict(nodes=[adjoint.centre_node(d)], dir=3, func=0, fscale=5.0),
                   dict(nodes=[mid], dir=2, skew=0, func=0, fscale=2.0)]
    return d


@pytest.mark.parametrize("resp", ["disp", "plastic"])
def test_adjoint_shfra_v4_skew_bcs_and_point_loads(resp):
    """ISHFRAM 2 element frames, a skewed /BCS edge (translations and a
    rotation) and time-function /CLOAD point loads, linear hardening: the
    adjoint against central differences along A, thickness and both."""
    need_gpu()
    n, p, N, STEP = 32, 2e6, 200, 1e-7
    wd, wpl = (1.0, 0.0) if resp == "disp" else (0.0, 1.0)
    A0, T0 = base_params(n)
    mk = lambda A, T: with_frame_skew_cloads(plate(n, A, T, p, N, jc_n=1.0))
    d0 = mk(A0, T0)
    node = adjoint.centre_node(d0)
    res = adjoint_run(d0, N, node, wd, wpl)
    J0, _ = forward_J(d0, N, node, wd, wpl)
    assert res["J"] == J0
    assert res["J"] > 0.0 if resp == "plastic" else res["J"] != 0.0
    gA, gT = res["dA"][0], adjoint.thickness_gradient(d0, res)[0]
    rng = np.random.default_rng(5)
    for name in ("A", "thk", "both"):
        uA = rng.choice([-1.0, 1.0], A0.size) if name in ("A", "both") else 0.0 * A0
        uT = rng.choice([-1.0, 1.0], T0.size) if name in ("thk", "both") else 0.0 * T0
        Jp, tp = forward_J(mk(A0 * (1 + STEP * uA), T0 * (1 + STEP * uT)), N, node, wd, wpl)
        Jm, tm = forward_J(mk(A0 * (1 - STEP * uA), T0 * (1 - STEP * uT)), N, node, wd, wpl)
        assert tp["tt"] == tm["tt"] == res["time"]["tt"]
        fd = (Jp - Jm) / (2 * STEP)
        ad = float(np.dot(gA, A0 * uA) + np.dot(gT, T0 * uT))
        assert abs(fd - ad) <= FD_REL * abs(ad), (name, fd, ad)


def test_adjoint_nodal_mass_gradient():
    """dJ/dMS along a random direction of the nodal masses (inertias fixed)."""
    need_gpu()
    from openradioss_b200.ecycle import ECycle
    n, p, N, STEP = 32, 2e6, 300, 1e-7
    A0, T0 = base_params(n)
    d0 = plate(n, A0, T0, p, N, jc_n=1.0)
    node = adjoint.centre_node(d0)
    res = adjoint_run(d0, N, node, 1.0, 0.0)
    ms0 = d0["parts"][0]["ms"].copy()
    u = np.random.default_rng(3).choice([-1.0, 1.0], ms0.size)
    Js = []
    for s in (+1, -1):
        d0["parts"][0]["ms"] = ms0 * (1 + s * STEP * u)
        Js.append(forward_J(d0, N, node, 1.0, 0.0)[0])
    d0["parts"][0]["ms"] = ms0
    fd = (Js[0] - Js[1]) / (2 * STEP)
    ad = float(np.dot(res["dms"][0], ms0 * u))
    assert abs(fd - ad) <= FD_REL * abs(ad), (fd, ad)


def test_adjoint_leaves_the_step_state_and_is_checkpoint_independent():
    """After or_ecycle_adjoint the handle holds what or_ecycle_step on the
    per-phase kernels would leave; the gradient does not depend on the
    checkpoint interval."""
    need_gpu()
    from openradioss_b200.ecycle import ECycle
    n, p, N = 32, 2e6, 120
    A0, T0 = base_params(n)
    d0 = plate(n, A0, T0, p, N)
    node = adjoint.centre_node(d0)
    r50 = adjoint_run(d0, N, node, 1.0, 0.5, checkpoint=50)
    r7 = adjoint_run(d0, N, node, 1.0, 0.5, checkpoint=7)
    for k in ("dA", "dthk", "dms", "din"):
        assert np.array_equal(r50[k][0], r7[k][0]), k
    h = ECycle(d0, precision=abi.OR_PREC_FP64, persistent=-1)
    h.step(N)
    ref = h.get_nodes()
    for k in ("x", "d", "v", "vr"):
        assert np.array_equal(ref[k], r50["nodes"][k]), k
    assert h.time() == r50["time"]
    e = h.energies()
    assert e == r50["energies"]
    h.close()


def test_gradcheck_harness():
    """torch.autograd.gradcheck (fast mode: one random unit direction) of the
    response as a function of relative changes of A and thickness, on the
    linear-hardening plate."""
    need_gpu()
    import torch
    n, p, N, STEP = 32, 2e6, 300, 1e-6
    A0, T0 = base_params(n)
    node = adjoint.centre_node(plate(n, A0, T0, p, N, jc_n=1.0))

    class PlateResponse(torch.autograd.Function):
        @staticmethod
        def forward(ctx, sA, sT):
            A = A0 * (1 + sA.detach().cpu().numpy())
            T = T0 * (1 + sT.detach().cpu().numpy())
            d = plate(n, A, T, p, N, jc_n=1.0)
            res = adjoint_run(d, N, node, 1.0, 1.0)
            ctx.gA = torch.tensor(res["dA"][0] * A, dtype=torch.float64)
            ctx.gT = torch.tensor(adjoint.thickness_gradient(d, res)[0] * T, dtype=torch.float64)
            return torch.tensor(res["J"], dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            return g * ctx.gA, g * ctx.gT

    sA = torch.zeros(A0.size, dtype=torch.float64, requires_grad=True)
    sT = torch.zeros(T0.size, dtype=torch.float64, requires_grad=True)
    J = PlateResponse.apply(sA, sT)
    J.backward()
    scale = float(torch.cat([sA.grad, sT.grad]).norm())
    assert torch.autograd.gradcheck(PlateResponse.apply, (sA.detach().requires_grad_(), sT.detach().requires_grad_()),
                                    eps=STEP, atol=1e-6 * scale, rtol=FD_REL, fast_mode=True,
                                    check_undefined_grad=False)
