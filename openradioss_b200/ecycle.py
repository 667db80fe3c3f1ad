"""Host-side binding of the C-ABI (include/or_ecycle.h) through ctypes.

``ECycle(deck, precision)`` uploads a deck (see ``openradioss_b200.decks``)
into one handle and exposes the same calls the Fortran RESOL loop makes:
``step(ncycles)``, ``get_nodes(part)``, ``hex_state(group)``,
``shell_state(group)``, ``energies(part)``.

The shared library ``libor_ecycle.so`` is built in-tree by
``openradioss_b200.build``; importing this module on a machine without it
raises, there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libor_ecycle.so")

_lib = None


def load_library(path: str = LIB_PATH):
    """Loads libor_ecycle.so; raises OSError if it has not been built."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise OSError(f"{path} not found: build it with `python -m openradioss_b200.build`")
    lib = C.CDLL(path)
    _declare(lib)
    if path == LIB_PATH:
        _lib = lib
    return lib


EXPORTS = [
    "or_ecycle_create", "or_ecycle_destroy", "or_ecycle_last_error", "or_ecycle_add_part",
    "or_ecycle_add_hex_group", "or_ecycle_add_shell_group", "or_ecycle_set_shell_yield",
    "or_ecycle_finalize", "or_ecycle_reset", "or_ecycle_step", "or_ecycle_get_nodes", "or_ecycle_set_nodes",
    "or_ecycle_get_hex_state", "or_ecycle_get_shell_state", "or_ecycle_energies",
    "or_ecycle_error_info", "or_ecycle_phase_times", "or_ecycle_launch_count",
    "or_ecycle_stream", "or_ecycle_device_bytes", "or_ecycle_adjoint", "or_ecycle_hex_step_noalloc",
    "or_ecycle_kernel_times", "or_ecycle_set_halo", "or_ecycle_spmd_buffer_bytes", "or_ecycle_spmd_begin",
    "or_ecycle_spmd_elements", "or_ecycle_spmd_nodes", "or_ecycle_spmd_end", "or_ecycle_add_rlink",
    "or_ecycle_set_rlink", "or_ecycle_add_function", "or_ecycle_add_cload", "or_ecycle_add_pload",
    "or_ecycle_add_skew", "or_ecycle_set_bcs_skew", "or_ecycle_set_hex_state", "or_ecycle_set_shell_state",
    "or_ecycle_set_energy_sums", "or_ecycle_persistent_info", "or_ecycle_add_rbody",
]


def _declare(lib):
    P = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    sig = {
        "or_ecycle_create": ([C.POINTER(abi.Config), C.POINTER(C.c_void_p)], C.c_int),
        "or_ecycle_destroy": ([P], C.c_int),
        "or_ecycle_last_error": ([P], C.c_char_p),
        "or_ecycle_add_part": ([P, C.c_int, dp, dp, dp, dp, dp, ip, ip, ip], C.c_int),
        "or_ecycle_add_hex_group": ([P, C.c_int, C.c_int, ip, C.POINTER(abi.Material),
                                     C.POINTER(abi.SolidProp), dp, ip], C.c_int),
        "or_ecycle_add_shell_group": ([P, C.c_int, C.c_int, ip, C.POINTER(abi.Material),
                                       C.POINTER(abi.ShellProp), dp, ip], C.c_int),
        "or_ecycle_set_shell_yield": ([P, C.c_int, dp], C.c_int),
        "or_ecycle_add_rlink": ([P, C.c_int, C.c_int, ip, C.c_int, C.c_int, ip], C.c_int),
        "or_ecycle_set_rlink": ([P, C.c_int, C.c_int, C.c_int], C.c_int),
        "or_ecycle_add_rbody": ([P, C.c_int, C.c_int, C.c_int, ip, dp, ip], C.c_int),
        "or_ecycle_add_function": ([P, C.c_int, dp, dp, ip], C.c_int),
        "or_ecycle_add_cload": ([P, C.c_int, C.c_int, ip, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, ip],
                                C.c_int),
        "or_ecycle_add_pload": ([P, C.c_int, C.c_int, ip, C.c_int, C.c_double, C.c_double, ip], C.c_int),
        "or_ecycle_add_skew": ([P, dp, ip], C.c_int),
        "or_ecycle_set_bcs_skew": ([P, C.c_int, ip], C.c_int),
        "or_ecycle_set_hex_state": ([P, C.c_int, dp, dp, dp, dp, dp, dp], C.c_int),
        "or_ecycle_set_shell_state": ([P, C.c_int, dp, dp, dp, dp, dp], C.c_int),
        "or_ecycle_set_energy_sums": ([P, C.c_int, C.c_double, C.c_double, C.c_double], C.c_int),
        "or_ecycle_finalize": ([P], C.c_int),
        "or_ecycle_reset": ([P], C.c_int),
        "or_ecycle_step": ([P, C.c_int, C.POINTER(abi.Time)], C.c_int),
        "or_ecycle_get_nodes": ([P, C.c_int, dp, dp, dp, dp], C.c_int),
        "or_ecycle_set_nodes": ([P, C.c_int, dp, dp, dp, dp], C.c_int),
        "or_ecycle_get_hex_state": ([P, C.c_int, dp, dp, dp, dp, dp, dp], C.c_int),
        "or_ecycle_get_shell_state": ([P, C.c_int, dp, dp, dp, dp, dp], C.c_int),
        "or_ecycle_energies": ([P, C.c_int, C.POINTER(abi.Energies)], C.c_int),
        "or_ecycle_error_info": ([P, ip, ip], C.c_int),
        "or_ecycle_phase_times": ([P, dp], C.c_int),
        "or_ecycle_launch_count": ([P, C.POINTER(C.c_longlong)], C.c_int),
        "or_ecycle_kernel_times": ([P, C.c_int, dp], C.c_int),
        "or_ecycle_set_halo": ([P, C.c_int, C.c_int, ip, ip, ip, C.c_int], C.c_int),
        "or_ecycle_spmd_buffer_bytes": ([P, C.POINTER(C.c_longlong)], C.c_int),
        "or_ecycle_spmd_begin": ([P, C.POINTER(abi.Time)], C.c_int),
        "or_ecycle_spmd_elements": ([P, P], C.c_int),
        "or_ecycle_spmd_nodes": ([P, P, C.c_int], C.c_int),
        "or_ecycle_spmd_end": ([P, C.POINTER(abi.Time)], C.c_int),
        "or_ecycle_stream": ([P, C.POINTER(C.c_void_p)], C.c_int),
        "or_ecycle_device_bytes": ([P, C.POINTER(C.c_longlong)], C.c_int),
        "or_ecycle_persistent_info": ([P, ip, ip, ip], C.c_int),
        "or_ecycle_adjoint": ([P, C.c_int, C.POINTER(abi.AdjointResponse), C.POINTER(abi.Time), dp, dp, dp, dp, dp],
                              C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res


class ECycleError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{abi.ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class _DeckModel:
    """Deck upload and accessors shared by the product handle and the CPU
    oracle binding; subclasses provide ``_call(name, *args)``."""

    def _load_deck(self, deck):
        self.deck = deck
        self.nparts = len(deck["parts"])
        self.hex_groups = []     # (part, nel)
        self.shell_groups = []   # (part, nel, npt)
        for f in deck.get("functions", []):
            fx, fy = _f64(f["x"]), _f64(f["y"])
            self._add_function(fx.size, fx, fy)
        for ax in deck.get("skews", []):
            self._add_skew(_f64(np.asarray(ax, np.float64).reshape(9)))
        for p in deck["parts"]:
            x, v, vr = _f64(p["x"]), _f64(p["v"]), _f64(p["vr"])
            ms, inr = _f64(p["ms"]), _f64(p["inr"])
            icodt, icodr = _i32(p["icodt"]), _i32(p["icodr"])
            part = self._add_part(x.shape[0], x, v, vr, ms, inr, icodt, icodr)
            for g in p["hex"]:
                ixs = _i32(g["ixs"])
                mat, prop = abi.make_material(g["mat"]), abi.make_solid_prop(g["prop"])
                vol0 = _f64(g["vol0"]) if g.get("vol0") is not None else None
                self._add_hex(part, ixs.shape[0], ixs, mat, prop, vol0)
                self.hex_groups.append((part, ixs.shape[0]))
            for g in p["shell"]:
                ixc = _i32(g["ixc"])
                mat, prop = abi.make_material(g["mat"]), abi.make_shell_prop(g["prop"])
                thke = _f64(g["thke"]) if g.get("thke") is not None else None
                gi = self._add_shell(part, ixc.shape[0], ixc, mat, prop, thke)
                if g.get("jc_a") is not None:
                    self._call("set_shell_yield", gi, abi.ptr(_f64(g["jc_a"]), C.c_double))
                self.shell_groups.append((part, ixc.shape[0], int(g["prop"]["npt"])))
            for rb in p.get("rbodies", []):
                sl = _i32(np.asarray(rb["slaves"]) + 1)
                self._add_rbody(part, int(rb["master"]) + 1, sl.size, sl, _f64(rb["rby"]))
            for rl in p.get("rlinks", []):
                nodes = _i32(np.asarray(rl["nodes"]) + 1)
                self._add_rlink(part, nodes.size, nodes, int(rl.get("ic", 7)), int(rl.get("icr", 0)))
            for cl in p.get("cloads", []):
                nodes = _i32(np.asarray(cl["nodes"]) + 1)
                self._add_cload(part, nodes.size, nodes, int(cl["dir"]), int(cl.get("skew", -1)), int(cl["func"]),
                                float(cl.get("ascale_x", 1.0)), float(cl.get("fscale", 1.0)))
            for pl in p.get("ploads", []):
                seg = _i32(np.asarray(pl["seg"]) + 1)          # -1 (triangle) -> 0
                self._add_pload(part, seg.shape[0], seg, int(pl["func"]), float(pl.get("ascale_x", 1.0)),
                                float(pl.get("fscale", 1.0)))
            if p.get("iskew") is not None:
                self._call("set_bcs_skew", part, abi.ptr(_i32(p["iskew"]), C.c_int))
        self._call("finalize")
        self.times = (abi.Time * self.nparts)(*[abi.initial_time() for _ in range(self.nparts)])

    def set_rlink(self, link, ic, icr=0):
        """New directions of rigid link ``link`` (0 and 0 switch it off)."""
        self._call("set_rlink", int(link), int(ic), int(icr))

    # --- accessors -----------------------------------------------------------
    def numnod(self, part=0):
        return self.deck["parts"][part]["x"].shape[0]

    def get_nodes(self, part=0):
        n = self.numnod(part)
        x, d, v, vr = (np.empty((n, 3)) for _ in range(4))
        self._call("get_nodes", part, *(abi.ptr(a, C.c_double) for a in (x, d, v, vr)))
        return dict(x=x, d=d, v=v, vr=vr)

    def hex_state(self, group):
        nel = self.hex_groups[group][1]
        sig = np.empty((6, nel))
        out = dict(sig=sig, eint=np.empty(nel), rho=np.empty(nel), qvis=np.empty(nel),
                   pla=np.empty(nel), epsd=np.empty(nel))
        self._call("get_hex_state", group, *(abi.ptr(out[k], C.c_double)
                                             for k in ("sig", "eint", "rho", "qvis", "pla", "epsd")))
        return out

    def shell_state(self, group):
        _, nel, npt = self.shell_groups[group]
        out = dict(sig=np.empty((npt, 5, nel)), pla=np.empty((npt, nel)), thk=np.empty(nel),
                   hourg=np.empty((3, nel)), eint=np.empty((2, nel)))
        self._call("get_shell_state", group, *(abi.ptr(out[k], C.c_double)
                                               for k in ("sig", "pla", "thk", "hourg", "eint")))
        return out

    def energies(self, part=0):
        e = abi.Energies()
        self._call("energies", part, C.byref(e))
        return dict(internal=e.internal, kinetic=e.kinetic, kinetic_rot=e.kinetic_rot,
                    hourglass=e.hourglass, plastic_work=e.plastic_work, external_work=e.external_work)

    def time(self, part=0):
        t = self.times[part]
        return dict(tt=t.tt, dt1=t.dt1, dt2=t.dt2, dt12=t.dt12, dt2old=t.dt2old, ncycle=t.ncycle,
                    ityptst=t.ityptst, neltst=t.neltst)


class ECycle(_DeckModel):
    """One device-resident handle (product path)."""

    def __init__(self, deck, precision=abi.OR_PREC_FP64, device=0, graph=1, lib=None, **cfg_kw):
        self.lib = lib or load_library()
        cfg = abi.make_config(precision=precision, device=device, graph=graph,
                              dtfac_solid=deck.get("dtfac_solid", 0.9),
                              dtfac_shell=deck.get("dtfac_shell", 0.9),
                              dtmx=deck.get("dtmx", 1e20), **cfg_kw)
        h = C.c_void_p()
        rc = self.lib.or_ecycle_create(C.byref(cfg), C.byref(h))
        if rc:
            raise ECycleError(rc, "or_ecycle_create failed")
        self.h = h
        self.precision = precision
        try:
            self._load_deck(deck)
        except Exception:
            self.close()
            raise

    def _call(self, name, *args):
        rc = getattr(self.lib, "or_ecycle_" + name)(self.h, *args)
        if rc:
            raise ECycleError(rc, self.lib.or_ecycle_last_error(self.h).decode())
        return rc

    def _add_part(self, n, x, v, vr, ms, inr, icodt, icodr):
        part = C.c_int()
        self._call("add_part", n, *(abi.ptr(a, C.c_double) for a in (x, v, vr, ms, inr)),
                   abi.ptr(icodt, C.c_int), abi.ptr(icodr, C.c_int), C.byref(part))
        return part.value

    def _add_hex(self, part, nel, ixs, mat, prop, vol0):
        g = C.c_int()
        self._call("add_hex_group", part, nel, abi.ptr(ixs, C.c_int), C.byref(mat), C.byref(prop),
                   abi.ptr(vol0, C.c_double), C.byref(g))
        return g.value

    def _add_shell(self, part, nel, ixc, mat, prop, thke):
        g = C.c_int()
        self._call("add_shell_group", part, nel, abi.ptr(ixc, C.c_int), C.byref(mat), C.byref(prop),
                   abi.ptr(thke, C.c_double), C.byref(g))
        return g.value

    def _add_rlink(self, part, n, nodes, ic, icr):
        li = C.c_int()
        self._call("add_rlink", part, n, abi.ptr(nodes, C.c_int), ic, icr, C.byref(li))
        return li.value

    def _add_rbody(self, part, master, n, slaves, rby):
        body = C.c_int()
        self._call("add_rbody", part, master, n, abi.ptr(slaves, C.c_int), abi.ptr(rby, C.c_double), C.byref(body))

    def _add_function(self, n, x, y):
        k = C.c_int()
        self._call("add_function", n, abi.ptr(x, C.c_double), abi.ptr(y, C.c_double), C.byref(k))

    def _add_skew(self, axes):
        k = C.c_int()
        self._call("add_skew", abi.ptr(axes, C.c_double), C.byref(k))

    def _add_cload(self, part, n, nodes, d, skew, func, ascale_x, fscale):
        k = C.c_int()
        self._call("add_cload", part, n, abi.ptr(nodes, C.c_int), d, skew, func, ascale_x, fscale, C.byref(k))

    def _add_pload(self, part, n, seg, func, ascale_x, fscale):
        k = C.c_int()
        self._call("add_pload", part, n, abi.ptr(seg, C.c_int), func, ascale_x, fscale, C.byref(k))

    def step(self, ncycles):
        self._call("step", int(ncycles), self.times)

    # --- restart -------------------------------------------------------------
    def set_nodes(self, part, x=None, d=None, v=None, vr=None):
        self._call("set_nodes", part, *(abi.ptr(_f64(a), C.c_double) if a is not None else None
                                       for a in (x, d, v, vr)))

    def set_hex_state(self, group, **state):
        keys = ("sig", "eint", "rho", "qvis", "pla", "epsd")
        arrs = [_f64(state[k]) if state.get(k) is not None else None for k in keys]
        self._call("set_hex_state", group, *(abi.ptr(a, C.c_double) for a in arrs))

    def set_shell_state(self, group, **state):
        keys = ("sig", "pla", "thk", "hourg", "eint")
        arrs = [_f64(state[k]) if state.get(k) is not None else None for k in keys]
        self._call("set_shell_state", group, *(abi.ptr(a, C.c_double) for a in arrs))

    def set_energy_sums(self, part, hourglass, plastic_work, external_work):
        self._call("set_energy_sums", part, float(hourglass), float(plastic_work), float(external_work))

    def restart_from(self, other):
        """Copies another handle's state (nodes, element state, time, energy
        sums) into this one, as a restart file would."""
        for p in range(self.nparts):
            n = other.get_nodes(p)
            self.set_nodes(p, n["x"], n["d"], n["v"], n["vr"])
            e = other.energies(p)
            self.set_energy_sums(p, e["hourglass"], e["plastic_work"], e["external_work"])
            self.times[p] = other.times[p]
        for gi in range(len(self.hex_groups)):
            self.set_hex_state(gi, **other.hex_state(gi))
        for gi in range(len(self.shell_groups)):
            self.set_shell_state(gi, **other.shell_state(gi))

    def reset(self):
        """Back to the uploaded initial state (nodes, elements, time, energies)."""
        self._call("reset")
        for p in range(self.nparts):
            self.times[p] = abi.initial_time()

    def error_info(self):
        code, idx = C.c_int(), C.c_int()
        self.lib.or_ecycle_error_info(self.h, C.byref(code), C.byref(idx))
        return code.value, idx.value

    def phase_times(self):
        a = np.zeros(4)
        self._call("phase_times", abi.ptr(a, C.c_double))
        return dict(hex=a[0], shell=a[1], node=a[2], total=a[3])

    def kernel_times(self, reps=64):
        """Device microseconds of one launch of each phase kernel (hex, shell,
        node), from graph-replayed back-to-back launches on the current state;
        the handle is reset afterwards."""
        a = np.zeros(3)
        self._call("kernel_times", int(reps), abi.ptr(a, C.c_double))
        for p in range(self.nparts):
            self.times[p] = abi.initial_time()
        return dict(hex=a[0], shell=a[1], node=a[2])

    def launch_count(self):
        n = C.c_longlong()
        self._call("launch_count", C.byref(n))
        return n.value

    def stream(self):
        s = C.c_void_p()
        self._call("stream", C.byref(s))
        return s.value

    def persistent_info(self):
        """(on, CTAs, threads per CTA) of the persistent form of step()."""
        on, g, t = C.c_int(), C.c_int(), C.c_int()
        self._call("persistent_info", C.byref(on), C.byref(g), C.byref(t))
        return bool(on.value), g.value, t.value

    def device_bytes(self):
        n = C.c_longlong()
        self._call("device_bytes", C.byref(n))
        return n.value

    def adjoint(self, ncycles, node=-1, comp=2, part=0, w_disp=1.0, w_plastic=0.0, checkpoint=50):
        """Runs ``ncycles`` like :meth:`step` and the reverse of those cycles
        (or_ecycle_adjoint).  Returns J = w_disp * D[node, comp] (end of the
        run) + w_plastic * (plastic work of the run) and its gradient with
        respect to the shell elements' Johnson-Cook A and initial thickness
        (one array per shell group) and the nodal masses and rotational
        inertias (one array per part), the dt sequence held fixed."""
        nsh = sum(g[1] for g in self.shell_groups)
        nno = sum(self.numnod(p) for p in range(self.nparts))
        dA, dthk, dms, din = np.zeros(nsh), np.zeros(nsh), np.zeros(nno), np.zeros(nno)
        J = C.c_double()
        r = abi.AdjointResponse(part, node, comp, checkpoint, w_disp, w_plastic)
        self._call("adjoint", int(ncycles), C.byref(r), self.times, C.byref(J),
                   *(abi.ptr(a, C.c_double) for a in (dA, dthk, dms, din)))
        gsplit = np.cumsum([g[1] for g in self.shell_groups])[:-1]
        nsplit = np.cumsum([self.numnod(p) for p in range(self.nparts)])[:-1]
        return dict(J=J.value, dA=np.split(dA, gsplit), dthk=np.split(dthk, gsplit),
                    dms=np.split(dms, nsplit), din=np.split(din, nsplit))

    def close(self):
        if getattr(self, "h", None):
            self.lib.or_ecycle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
