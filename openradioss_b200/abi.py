"""ctypes mirrors of the structs declared in include/or_ecycle.h."""
from __future__ import annotations

import ctypes as C

OR_OK = 0
OR_E_ARG = 1
OR_E_CUDA = 2
OR_E_STATE = 3
OR_E_NEGVOL = 4
OR_E_DTMIN = 5
OR_E_NAN = 6
OR_E_TIMEOUT = 7
OR_E_UNSUPPORTED = 8
OR_E_NOMEM = 9

OR_PREC_FP64 = 0
OR_PREC_SPLIT = 1

ERROR_NAMES = {
    OR_E_ARG: "bad argument", OR_E_CUDA: "CUDA error", OR_E_STATE: "call out of order",
    OR_E_NEGVOL: "negative volume", OR_E_DTMIN: "time step below DTMIN",
    OR_E_NAN: "NaN in nodal acceleration", OR_E_TIMEOUT: "timeout",
    OR_E_UNSUPPORTED: "unsupported option", OR_E_NOMEM: "out of device memory",
}


class Config(C.Structure):
    _fields_ = [("precision", C.c_int), ("device", C.c_int),
                ("dtfac_solid", C.c_double), ("dtfac_shell", C.c_double),
                ("dtmin_solid", C.c_double), ("dtmin_shell", C.c_double),
                ("dtmx", C.c_double), ("dt_growth", C.c_double),
                ("graph", C.c_int), ("block_hex", C.c_int), ("block_shell", C.c_int),
                ("block_node", C.c_int), ("persistent", C.c_int)]


class Material(C.Structure):
    _fields_ = [("law", C.c_int), ("rho0", C.c_double), ("young", C.c_double), ("nu", C.c_double),
                ("shear", C.c_double), ("bulk", C.c_double), ("a11", C.c_double), ("a12", C.c_double),
                ("ssp_shell", C.c_double), ("jc_a", C.c_double), ("jc_b", C.c_double),
                ("jc_n", C.c_double), ("epsmax", C.c_double), ("sigmax", C.c_double)]


class SolidProp(C.Structure):
    _fields_ = [("qa", C.c_double), ("qb", C.c_double), ("qh", C.c_double), ("jcvt", C.c_int), ("pad", C.c_int)]


class ShellProp(C.Structure):
    _fields_ = [("thk", C.c_double), ("npt", C.c_int), ("ithk", C.c_int), ("ipla", C.c_int),
                ("ishfram", C.c_int), ("hm", C.c_double), ("hf", C.c_double), ("hr", C.c_double), ("shf", C.c_double),
                ("pressure", C.c_double), ("dn", C.c_double), ("ishell", C.c_int), ("pad", C.c_int)]


class Time(C.Structure):
    _fields_ = [("tt", C.c_double), ("dt1", C.c_double), ("dt2", C.c_double), ("dt12", C.c_double),
                ("dt2old", C.c_double), ("ncycle", C.c_int), ("ityptst", C.c_int),
                ("neltst", C.c_int), ("pad", C.c_int)]


class Energies(C.Structure):
    _fields_ = [("internal", C.c_double), ("kinetic", C.c_double), ("kinetic_rot", C.c_double),
                ("hourglass", C.c_double), ("plastic_work", C.c_double), ("external_work", C.c_double)]


class AdjointResponse(C.Structure):
    _fields_ = [("part", C.c_int), ("node", C.c_int), ("comp", C.c_int), ("checkpoint", C.c_int),
                ("w_disp", C.c_double), ("w_plastic", C.c_double)]


# the growth factor of resol.F:6080 is the default-REAL literal 1.1
DT_GROWTH_REF = float(__import__("numpy").float32(1.1))


def make_config(precision=OR_PREC_FP64, device=0, dtfac_solid=0.9, dtfac_shell=0.9,
                dtmx=1e20, graph=1, block_hex=0, block_shell=0, block_node=0,
                dtmin_solid=0.0, dtmin_shell=0.0, persistent=0):
    return Config(precision, device, dtfac_solid, dtfac_shell, dtmin_solid, dtmin_shell, dtmx,
                  DT_GROWTH_REF, graph, block_hex, block_shell, block_node, persistent)


def make_material(m: dict) -> Material:
    return Material(int(m["law"]), m["rho0"], m["young"], m["nu"], m["shear"], m["bulk"], m["a11"],
                    m["a12"], m["ssp_shell"], m["jc_a"], m["jc_b"], m["jc_n"], m["epsmax"], m["sigmax"])


def make_solid_prop(p: dict) -> SolidProp:
    return SolidProp(p["qa"], p["qb"], p["qh"], int(p.get("jcvt", 0)), 0)


def make_shell_prop(p: dict) -> ShellProp:
    return ShellProp(p["thk"], int(p["npt"]), int(p["ithk"]), int(p["ipla"]), int(p.get("ishfram", 0)),
                     p["hm"], p["hf"], p["hr"], p["shf"], p["pressure"], float(p.get("dn", 0.0)),
                     int(p.get("ishell", 1)), 0)


def initial_time(dt2old=1e30):
    """RESOL state before the first cycle: DT2 = 0 so that the first element
    pass runs with DT1 = 0, no growth cap (DT2OLD large)."""
    return Time(0.0, 0.0, 0.0, 0.0, dt2old, 0, 0, -1, 0)


def ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None
