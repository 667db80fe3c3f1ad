"""ctypes binding of the CPU oracle (test infrastructure only).

The oracle is a C++ restatement of the reference Fortran element cycle
(ecycle_oracle.cpp); it is the parity checker for the CUDA path and the CPU
baseline of bench.py.  It shares the deck format and the accessors of the
product binding, so a test drives both with the same code.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

from openradioss_b200 import abi
from openradioss_b200.ecycle import ECycleError, _DeckModel

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PARITY = os.path.join(HERE, "liboracle_ecycle.so")
LIB_FAST = os.path.join(HERE, "liboracle_ecycle_fast.so")


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load(fast=False):
    path = LIB_FAST if fast else LIB_PARITY
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    lib.oracle_create.argtypes = [C.POINTER(abi.Config)]
    lib.oracle_create.restype = P
    lib.oracle_destroy.argtypes = [P]
    lib.oracle_add_part.argtypes = [P, C.c_int, dp, dp, dp, dp, dp, ip, ip]
    lib.oracle_add_hex_group.argtypes = [P, C.c_int, C.c_int, ip, C.POINTER(abi.Material),
                                         C.POINTER(abi.SolidProp), dp]
    lib.oracle_add_shell_group.argtypes = [P, C.c_int, C.c_int, ip, C.POINTER(abi.Material),
                                           C.POINTER(abi.ShellProp), dp]
    lib.oracle_set_shell_yield.argtypes = [P, C.c_int, dp]
    lib.oracle_add_rlink.argtypes = [P, C.c_int, C.c_int, ip, C.c_int, C.c_int]
    lib.oracle_set_rlink.argtypes = [P, C.c_int, C.c_int, C.c_int]
    lib.oracle_add_rbody.argtypes = [P, C.c_int, C.c_int, C.c_int, ip, dp]
    lib.oracle_add_function.argtypes = [P, C.c_int, dp, dp]
    lib.oracle_add_cload.argtypes = [P, C.c_int, C.c_int, ip, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double]
    lib.oracle_add_pload.argtypes = [P, C.c_int, C.c_int, ip, C.c_int, C.c_double, C.c_double]
    lib.oracle_add_skew.argtypes = [P, dp]
    lib.oracle_set_bcs_skew.argtypes = [P, C.c_int, ip]
    lib.oracle_finalize.argtypes = [P]
    lib.oracle_step.argtypes = [P, C.c_int, C.POINTER(abi.Time), C.c_int]
    lib.oracle_get_nodes.argtypes = [P, C.c_int, dp, dp, dp, dp]
    lib.oracle_get_hex_state.argtypes = [P, C.c_int, dp, dp, dp, dp, dp, dp]
    lib.oracle_get_shell_state.argtypes = [P, C.c_int, dp, dp, dp, dp, dp]
    lib.oracle_energies.argtypes = [P, C.c_int, C.POINTER(abi.Energies)]
    lib.oracle_error_info.argtypes = [P, ip, ip]
    return lib


class Oracle(_DeckModel):
    def __init__(self, deck, precision=abi.OR_PREC_FP64, nthreads=1, fast=False):
        self.lib = load(fast)
        cfg = abi.make_config(precision=precision, dtfac_solid=deck.get("dtfac_solid", 0.9),
                              dtfac_shell=deck.get("dtfac_shell", 0.9), dtmx=deck.get("dtmx", 1e20))
        self.h = self.lib.oracle_create(C.byref(cfg))
        self.nthreads = nthreads
        self.precision = precision
        self._nhex = 0
        self._nshell = 0
        self._load_deck(deck)

    def _call(self, name, *args):
        rc = getattr(self.lib, "oracle_" + name)(self.h, *args)
        if rc:
            code, idx = C.c_int(), C.c_int()
            self.lib.oracle_error_info(self.h, C.byref(code), C.byref(idx))
            raise ECycleError(rc, f"oracle {name} failed at index {idx.value}")
        return rc

    def _add_part(self, n, x, v, vr, ms, inr, icodt, icodr):
        self._call("add_part", n, *(abi.ptr(a, C.c_double) for a in (x, v, vr, ms, inr)),
                   abi.ptr(icodt, C.c_int), abi.ptr(icodr, C.c_int))
        return self._count_part()

    def _count_part(self):
        self._np = getattr(self, "_np", 0) + 1
        return self._np - 1

    def _add_hex(self, part, nel, ixs, mat, prop, vol0):
        self._call("add_hex_group", part, nel, abi.ptr(ixs, C.c_int), C.byref(mat), C.byref(prop),
                   abi.ptr(vol0, C.c_double))
        self._nhex += 1
        return self._nhex - 1

    def _add_shell(self, part, nel, ixc, mat, prop, thke):
        self._call("add_shell_group", part, nel, abi.ptr(ixc, C.c_int), C.byref(mat), C.byref(prop),
                   abi.ptr(thke, C.c_double))
        self._nshell += 1
        return self._nshell - 1

    def _add_rlink(self, part, n, nodes, ic, icr):
        self._call("add_rlink", part, n, abi.ptr(nodes, C.c_int), ic, icr)

    def _add_rbody(self, part, master, n, slaves, rby):
        self._call("add_rbody", part, master, n, abi.ptr(slaves, C.c_int), abi.ptr(rby, C.c_double))

    def _add_function(self, n, x, y):
        self._call("add_function", n, abi.ptr(x, C.c_double), abi.ptr(y, C.c_double))

    def _add_skew(self, axes):
        self._call("add_skew", abi.ptr(axes, C.c_double))

    def _add_cload(self, part, n, nodes, d, skew, func, ascale_x, fscale):
        self._call("add_cload", part, n, abi.ptr(nodes, C.c_int), d, skew, func, ascale_x, fscale)

    def _add_pload(self, part, n, seg, func, ascale_x, fscale):
        self._call("add_pload", part, n, abi.ptr(seg, C.c_int), func, ascale_x, fscale)

    def step(self, ncycles):
        self._call("step", int(ncycles), self.times, self.nthreads)

    def error_info(self):
        code, idx = C.c_int(), C.c_int()
        self.lib.oracle_error_info(self.h, C.byref(code), C.byref(idx))
        return code.value, idx.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
