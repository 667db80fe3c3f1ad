"""Shell element adjoint against central finite differences, on the CPU.

The element reverse used by the GPU adjoint (openradioss_b200/csrc/shell_adjoint.cuh)
is compiled here for the host with g++ and checked on random element states:
for random output weights w and a random input direction u,

    (w . out(in + h u) - w . out(in - h u)) / 2h   ==   reverse(w) . u

per input group (coordinates, velocities, rotational velocities, stresses,
plastic strains, thickness, hourglass history, Johnson-Cook A), on the elastic
and plastic branches of the radial return, LAW1 and LAW2, ITHK 0 and 1, with
and without pressure, for a degenerate (triangular) quad, and in the /SHFRA/V4
(ISHFRAM 2) frame.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "adjoint_host", "shell_adjoint_host.cpp")

NIN, NOUT = 103, 89
SL = dict(x=slice(0, 12), v=slice(12, 24), vr=slice(24, 36), sig=slice(36, 86), pla=slice(86, 96),
          thk=slice(96, 97), thke=slice(97, 98), hourg=slice(98, 101), ca=slice(101, 102), dt1=slice(102, 103))
OSL = dict(f=slice(0, 12), m=slice(12, 24), sig=slice(24, 74), pla=slice(74, 84), thk=slice(84, 85),
           hourg=slice(85, 88), wpla=slice(88, 89))


class ShellParams(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("law", "npt", "ithk", "degen", "ishfram", "pad")] + \
               [(n, C.c_double) for n in ("rho", "young", "nu", "shear", "a11", "a12", "jc_b", "jc_n", "sigmax",
                                          "hm", "hf", "hr", "shf", "pressure")]


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    so = str(tmp_path_factory.mktemp("adj") / "libshell_adjoint_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-ffp-contract=off", "-o", so, SRC], check=True)
    L = C.CDLL(so)
    dp = C.POINTER(C.c_double)
    L.adj_forward.argtypes = [C.POINTER(ShellParams), dp, dp]
    L.adj_reverse.argtypes = [C.POINTER(ShellParams), dp, dp, dp]
    nin, nout = C.c_int(), C.c_int()
    assert L.adj_sizes(C.byref(nin), C.byref(nout)) == 10
    assert (nin.value, nout.value) == (NIN, NOUT)
    return L


def params(law=2, npt=5, ithk=1, degen=0, pressure=2e6, ishfram=0):
    E, nu, rho = 70e9, 0.33, 2700.0
    G = E / (2 * (1 + nu))
    return ShellParams(law=law, npt=npt, ithk=ithk, degen=degen, ishfram=ishfram, pad=0, rho=rho, young=E, nu=nu,
                       shear=G,
                       a11=E / (1 - nu * nu), a12=E * nu / (1 - nu * nu), jc_b=275e6, jc_n=0.36, sigmax=1e30,
                       hm=0.01, hf=0.01, hr=0.01, shf=5.0 / 6.0, pressure=pressure)


def random_input(rng, sig_scale, pla_mode, degen=False):
    h = 1e-3
    x = np.array([[0, 0, 0], [h, 0, 0], [h, h, 0], [0, h, 0]], float)
    x[:, :2] += rng.uniform(-0.1, 0.1, (4, 2)) * h
    x[:, 2] += rng.uniform(-0.05, 0.05, 4) * h
    if degen:
        x[3] = x[2]
    a = np.zeros(NIN)
    a[SL["x"]] = x.ravel()
    a[SL["v"]] = rng.normal(0, 1.0, 12)
    a[SL["vr"]] = rng.normal(0, 100.0, 12)
    a[SL["sig"]] = rng.normal(0, sig_scale, 50)
    if pla_mode == "zero":
        a[SL["pla"]] = 0.0
    else:
        a[SL["pla"]] = rng.uniform(0.005, 0.02, 10)
    a[SL["thk"]] = 1.0e-3
    a[SL["thke"]] = 1.02e-3
    a[SL["hourg"]] = rng.normal(0, 1e-2, 3)
    a[SL["ca"]] = 350e6
    a[SL["dt1"]] = 1.5e-7
    return a


IN_SCALE = dict(x=1e-3, v=1.0, vr=100.0, sig=1e8, pla=1e-2, thk=1e-3, thke=1e-3, hourg=1e-2, ca=3.5e8)
OUT_SCALE = dict(f=1e2, m=1e-1, sig=1e8, pla=1e-2, thk=1e-3, hourg=1e-2, wpla=1e-5)


def fwd(L, P, a):
    out = np.zeros(NOUT)
    L.adj_forward(C.byref(P), a.ctypes.data_as(C.POINTER(C.c_double)), out.ctypes.data_as(C.POINTER(C.c_double)))
    return out


def rev(L, P, a, w):
    ib = np.zeros(NIN)
    L.adj_reverse(C.byref(P), a.ctypes.data_as(C.POINTER(C.c_double)), w.ctypes.data_as(C.POINTER(C.c_double)),
                  ib.ctypes.data_as(C.POINTER(C.c_double)))
    return ib


def check(L, P, a, rng, groups=IN_SCALE, rel=1e-6, h=1e-6):
    npt = P.npt
    w = np.zeros(NOUT)
    for k, s in OUT_SCALE.items():
        w[OSL[k]] = rng.normal(0, 1.0, OSL[k].stop - OSL[k].start) / s
    # only the first npt integration points exist
    w[OSL["sig"]][5 * npt:] = 0.0
    w[OSL["pla"]][npt:] = 0.0
    ib = rev(L, P, a, w)
    worst = {}
    for g, s in groups.items():
        u = np.zeros(NIN)
        n = SL[g].stop - SL[g].start
        u[SL[g]] = rng.normal(0, 1.0, n) * s
        if g == "sig":
            u[SL[g]][5 * npt:] = 0.0
        if g == "pla":
            u[SL[g]][npt:] = 0.0
        if g == "x" and P.degen:
            u[9:12] = u[6:9]            # keep the triangle degenerate
        op, om = fwd(L, P, a + h * u), fwd(L, P, a - h * u)
        fd = (w @ op - w @ om) / (2 * h)
        ad = ib @ u
        # rounding floor of the difference quotient: a few ulps of sum |w_i out_i| over 2h
        floor = 64 * np.finfo(float).eps * np.abs(w * op).sum() / (2 * h)
        worst[g] = (abs(fd - ad) / (rel * max(abs(fd), abs(ad)) + floor), fd, ad)
    bad = {g: v for g, v in worst.items() if v[0] > 1.0}
    assert not bad, f"adjoint vs FD mismatch: {bad}"
    return worst


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_law2_plastic_pressure(lib, seed):
    rng = np.random.default_rng(seed)
    P = params(law=2, npt=5, ithk=1, pressure=2e6)
    a = random_input(rng, 4e8, "pos")
    out = fwd(lib, P, a)
    assert out[OSL["wpla"]][0] > 0.0          # plastic branch taken
    check(lib, P, a, rng)


@pytest.mark.parametrize("seed", [3, 4])
def test_law2_elastic(lib, seed):
    rng = np.random.default_rng(seed)
    P = params(law=2, npt=5, ithk=1, pressure=0.0)
    a = random_input(rng, 2e7, "pos")
    out = fwd(lib, P, a)
    assert out[OSL["wpla"]][0] == 0.0
    check(lib, P, a, rng)


def test_law2_first_yield_from_zero_plastic_strain(lib):
    rng = np.random.default_rng(5)
    P = params(law=2, npt=5, ithk=1)
    a = random_input(rng, 4e8, "zero")
    assert fwd(lib, P, a)[OSL["wpla"]][0] > 0.0
    check(lib, P, a, rng, groups={k: v for k, v in IN_SCALE.items() if k != "pla"})


@pytest.mark.parametrize("npt", [1, 3])
def test_law1_ithk0(lib, npt):
    rng = np.random.default_rng(10 + npt)
    P = params(law=1, npt=npt, ithk=0, pressure=1e6)
    a = random_input(rng, 1e8, "pos")
    w = check(lib, P, a, rng)
    assert abs(w["thke"][2]) > 0.0            # THKE is the thickness used when ITHK = 0


def test_degenerate_triangle(lib):
    rng = np.random.default_rng(7)
    P = params(law=2, npt=5, ithk=1, degen=1)
    a = random_input(rng, 4e8, "pos", degen=True)
    check(lib, P, a, rng)


@pytest.mark.parametrize("seed", [20, 21])
def test_shfra_v4_frame(lib, seed):
    """ISHFRAM 2 (/SHFRA/V4) frame, plastic branch, with a warped quad."""
    rng = np.random.default_rng(seed)
    P = params(law=2, npt=5, ithk=1, ishfram=2)
    a = random_input(rng, 4e8, "pos")
    assert fwd(lib, P, a)[OSL["wpla"]][0] > 0.0
    check(lib, P, a, rng)
    # the frame matters: the same element in the default frame gives other forces
    P0 = params(law=2, npt=5, ithk=1, ishfram=0)
    assert not np.allclose(fwd(lib, P, a)[OSL["f"]], fwd(lib, P0, a)[OSL["f"]], rtol=1e-9, atol=0)
