"""FP64 reference gradient of a shell run, on the CPU (test infrastructure).

The forward states come from the oracle (FP64), one cycle at a time.  The
reverse of each cycle is restated here in numpy, in the order the cycle runs
backwards:
- DEPLA / VELOCITY / BCS10 / ACCELE of every node (global codes only):
  V(n+1) = V(n) + DT12 F / MS on free components, 0 on fixed ones, and
  X, D += DT2 V(n+1); the same for VR with the moments and IN;
- then every element through the element reverse of
  openradioss_b200/csrc/shell_adjoint.cuh, compiled for the host by
  tests/adjoint_host/shell_adjoint_host.cpp (it recomputes the element forward
  from the stored state and runs the reverse), its corner adjoints added to
  the nodes.
The time-step sequence is the forward's, held fixed.  The element reverse is
the same code the GPU runs (checked on its own against central differences in
test_shell_adjoint_fd.py); the nodal reverse, the corner assembly and the
checkpointing are independent of the GPU's.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from openradioss_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "adjoint_host", "shell_adjoint_host.cpp")
NIN, NOUT, NPMAX = 103, 89, 10


class ShellParams(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("law", "npt", "ithk", "degen", "ishfram", "pad")] + \
               [(n, C.c_double) for n in ("rho", "young", "nu", "shear", "a11", "a12", "jc_b", "jc_n", "sigmax",
                                          "hm", "hf", "hr", "shf", "pressure")]


def build_host_lib(outdir):
    so = os.path.join(str(outdir), "libshell_adjoint_ref.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", so, SRC], check=True)
    lib = C.CDLL(so)
    dp = C.POINTER(C.c_double)
    lib.adj_reverse.argtypes = [C.POINTER(ShellParams), dp, dp, dp]
    lib.adj_forward.argtypes = [C.POINTER(ShellParams), dp, dp]
    return lib


def group_params(g):
    """The element parameters of a shell group, as the handle derives them."""
    m, p = abi.make_material(g["mat"]), abi.make_shell_prop(g["prop"])
    return ShellParams(law=m.law, npt=p.npt, ithk=p.ithk, degen=0, ishfram=p.ishfram, pad=0, rho=m.rho0,
                       young=m.young, nu=m.nu, shear=m.shear, a11=m.a11, a12=m.a12, jc_b=m.jc_b, jc_n=m.jc_n,
                       sigmax=m.sigmax, hm=p.hm, hf=p.hf, hr=p.hr, shf=p.shf, pressure=p.pressure)


def reference_gradient(deck, ncycles, node, comp, w_disp, w_plastic, lib):
    """J and dJ/dA, dJ/dthk (direct), dJ/dMS, dJ/dIN of a one-part, one-shell-group
    deck, in the dict layout of ECycle.adjoint."""
    from oracle.oracle import Oracle
    P = deck["parts"][0]
    g = P["shell"][0]
    if len(deck["parts"]) != 1 or len(P["shell"]) != 1 or P["hex"]:
        raise ValueError("one part with one shell group")
    conn = np.asarray(g["ixc"])[:, 1:5] - 1
    nel, nn = conn.shape[0], P["x"].shape[0]
    prm = group_params(g)
    npt = prm.npt
    thk0 = float(g["prop"]["thk"])
    thke = np.asarray(g["thke"], float) if g.get("thke") is not None else np.full(nel, thk0)
    ca = np.asarray(g["jc_a"], float) if g.get("jc_a") is not None else np.full(nel, float(g["mat"]["jc_a"]))
    ms, inr = np.asarray(P["ms"], float), np.asarray(P["inr"], float)
    icodt, icodr = np.asarray(P["icodt"]), np.asarray(P["icodr"])
    tfix = np.stack([(icodt & 4) != 0, (icodt & 2) != 0, (icodt & 1) != 0], axis=1)
    rfix = np.stack([(icodr & 4) != 0, (icodr & 2) != 0, (icodr & 1) != 0], axis=1)

    o = Oracle(deck, precision=abi.OR_PREC_FP64)
    wp0 = o.energies()["plastic_work"]
    rec = []
    for _ in range(ncycles):
        rec.append((o.get_nodes(), o.shell_state(0), o.time()))
        o.step(1)
    end = (o.get_nodes(), None, o.time())
    J = w_disp * end[0]["d"][node, comp] + w_plastic * (o.energies()["plastic_work"] - wp0)
    o.close()

    lX, lD, lV, lR = (np.zeros((nn, 3)) for _ in range(4))
    lD[node, comp] = w_disp
    lsig, lpla = np.zeros((npt, 5, nel)), np.zeros((npt, nel))
    lthk, lh = np.zeros(nel), np.zeros((3, nel))
    dA, dthke, dms, din = np.zeros(nel), np.zeros(nel), np.zeros(nn), np.zeros(nn)
    xin, xob, xib = (np.zeros(k) for k in (NIN, NOUT, NIN))
    ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    for n in reversed(range(ncycles)):
        nd, st, t0 = rec[n]
        nd1, t1 = (rec[n + 1][0], rec[n + 1][2]) if n + 1 < ncycles else (end[0], end[2])
        DT2, DT12 = t1["dt2"], t1["dt12"]
        # nodes: V(n+1) = V(n) + DT12 F / MS (free), X and D += DT2 V(n+1)
        bar = lV + DT2 * (lX + lD)
        bar[tfix] = 0.0
        lA = DT12 * bar
        A = (nd1["v"] - nd["v"]) / DT12
        pos = ms > 0
        lF = np.zeros((nn, 3))
        lF[pos] = lA[pos] / ms[pos, None]
        dms[pos] -= (lA[pos] * A[pos]).sum(axis=1) / ms[pos]
        barR = lR.copy()
        barR[rfix] = 0.0
        lAR = DT12 * barR
        AR = (nd1["vr"] - nd["vr"]) / DT12
        pr = inr > 0
        lM = np.zeros((nn, 3))
        lM[pr] = lAR[pr] / inr[pr, None]
        din[pr] -= (lAR[pr] * AR[pr]).sum(axis=1) / inr[pr]
        nX, nV, nR = lX.copy(), bar, barR
        # elements
        for e in range(nel):
            c = conn[e]
            prm.degen = 1 if c[2] == c[3] else 0
            xin[:] = 0.0
            xin[0:12] = nd["x"][c].ravel()
            xin[12:24] = nd["v"][c].ravel()
            xin[24:36] = nd["vr"][c].ravel()
            xin[36:36 + 5 * npt] = st["sig"][:, :, e].ravel()
            xin[86:86 + npt] = st["pla"][:, e]
            xin[96], xin[97] = st["thk"][e], thke[e]
            xin[98:101] = st["hourg"][:, e]
            xin[101], xin[102] = ca[e], t0["dt2"]
            xob[:] = 0.0
            xob[0:12] = lF[c].ravel()
            xob[12:24] = lM[c].ravel()
            xob[24:24 + 5 * npt] = lsig[:, :, e].ravel()
            xob[74:74 + npt] = lpla[:, e]
            xob[84] = lthk[e]
            xob[85:88] = lh[:, e]
            xob[88] = w_plastic
            xib[:] = 0.0
            lib.adj_reverse(C.byref(prm), ptr(xin), ptr(xob), ptr(xib))
            # corners in ascending order: a node shared by two corners gets both
            for k in range(4):
                nX[c[k]] += xib[3 * k:3 * k + 3]
                nV[c[k]] += xib[12 + 3 * k:12 + 3 * k + 3]
                nR[c[k]] += xib[24 + 3 * k:24 + 3 * k + 3]
            lsig[:, :, e] = xib[36:36 + 5 * npt].reshape(npt, 5)
            lpla[:, e] = xib[86:86 + npt]
            lthk[e] = xib[96]
            dthke[e] += xib[97]
            lh[:, e] = xib[98:101]
            dA[e] += xib[101]
        lX, lV, lR = nX, nV, nR
    return dict(J=J, dA=[dA], dthk=[lthk + dthke], dms=[dms], din=[din])
