"""Reader of Radioss block-format input decks for the element-cycle path.

A reference run is a starter deck (``<run>_0000.rad``) followed by one or more
engine decks (``<run>_0001.rad``, ...).  This module reads the keywords that
define what the element cycle computes and turns them into the deck dict of
:mod:`openradioss_b200.decks` (one part holding every node), with the starter's
nodal masses and inertias:

starter keywords
  /BEGIN (input version >= 2017: 20-character real fields), /NODE,
  /SHELL/<part>, /BRICK/<part>, /PART, /PROP/SHELL (TYPE1), /PROP/SOLID
  (TYPE14, Isolid 1, Iframe 1 or 2, Ismstr 4), /MAT/PLAS_JOHNS (LAW2, Iflag 0),
  /MAT/ELAST (LAW1), /DEF_SHELL, /DEF_SOLID, /SHFRA/V4, /SKEW/FIX, /BCS,
  /GRNOD/NODE, /INIVEL/TRA (no skew), /ADMAS/0, /FUNCT, /CLOAD (time
  abscissa, no sensor), /PLOAD (no sensor), /SURF/SEG, /SURF/PART (shell parts)
engine keywords
  /RUN (final time), /VEL/TRA and /VEL/ROT (rigid velocity links, no skew)

Keywords that only request output (/TITLE, /TH, /ANIM, /PRINT, ...) are
skipped; any other keyword raises :class:`RadError`, so a deck is never run
with part of its physics silently dropped.

Starter semantics restated here (the reference starter is not on the path):

* /PROP/SHELL flags fall back to /DEF_SHELL, then to the built-in defaults
  Ishell 1, Ismstr 2, Ithick 0, Iplas 0 (hm_read_prop01.F:112-272,
  defaults_mod.F90:160-165); Ishell 1 to 4 are read (the library maps them to
  the engine's IHBE 1, 0, 2, 4); hm = hf = 0.1, hr = 0.01 when zero for
  Ishell 3, hm = hf = hr = 0.01 otherwise, and shear factor 5/6
  (hm_read_prop01.F:204-240); Dn is kept for one-point shells (MHVIS3);
* global integration N = 0 with LAW2 becomes 3 integration points
  (cgrtails.F:795-806, warning 1912); LAW1 keeps N = 0 only with the
  resultant law, which the element cycle does not implement;
* shell nodal mass rho t A / 4 and inertia EMS (A / 9 + t^2 / 12), with A the
  CEVECI area 1/2 |(x3 - x1) x (x4 - x2)| (cinmas.F:369, :703; ceveci.F);
  hexa nodal mass rho0 V0 / 8 (smass3.F:79-94); /ADMAS type 0 adds its mass to
  every node of the group;
* /PROP/SOLID: Isolid, Ismstr, Iframe fall back to /DEF_SOLID, then to 1, 4, 1;
  qa = 1.1, qb = 0.05, h = 0.1 when zero (hm_read_prop14.F:218-380);
* /SKEW/FIX: x' = Y x Z, y' = Z x x', all three normalised (hm_read_skw.F);
* /CLOAD and /PLOAD: Ascale_x and Fscale_y default to 1 (hm_read_cload.F,
  hm_read_pload.F);
* LAW2: G = E / 2(1 + nu), A11 = E / (1 - nu^2), shell sound speed
  sqrt(E / rho) (hm_read_mat02_jc.F90); SIG_max0 = 0 and EPS_p_max = 0 mean
  no limit.
"""
from __future__ import annotations

import math
import os

import numpy as np

from . import decks


class RadError(ValueError):
    """Deck outside what the reader (and the element cycle) implements."""


# keywords that only steer output, restart files or the reference's own
# parallel setup; they do not change the element cycle
_IGNORED_STARTER = {"TITLE", "ANALY", "IOFLAG", "SPMD", "TH", "END", "RANDOM"}
_IGNORED_ENGINE = {"ANIM", "PRINT", "TFILE", "MON", "VERS", "PROC", "H3D", "OUTP", "RFILE", "PARITH",
                   "STOP", "TITLE", "END"}


def _int(line, col, width=10, default=0):
    s = line[col:col + width].strip()
    return int(s) if s else default


def _real(line, col, width=20, default=0.0):
    s = line[col:col + width].strip()
    if not s:
        return default
    s = s.replace("D", "E").replace("d", "e")
    # Fortran reals may omit the exponent letter: "1.5-3"
    for i in range(1, len(s)):
        if s[i] in "+-" and s[i - 1] not in "eE" and s[i - 1].isdigit():
            s = s[:i] + "e" + s[i:]
            break
    return float(s)


def _blocks(path):
    """(keyword fields, data lines, line number) of every block of a deck;
    comment lines (#, $) dropped, ``#include`` followed relative to the deck."""
    base = os.path.dirname(os.path.abspath(path))
    out = []
    cur = None

    def feed(p):
        nonlocal cur
        with open(p, "r", errors="replace") as f:
            for ln, raw in enumerate(f, 1):
                line = raw.rstrip("\n\r")
                if line.startswith("#include"):
                    feed(os.path.join(base, line.split(None, 1)[1].strip()))
                    continue
                if not line.strip() or line[0] in "#$":
                    continue
                if line[0] == "/":
                    cur = ([k for k in line.strip()[1:].split("/") if k != ""], [], (p, ln))
                    out.append(cur)
                elif cur is not None:
                    cur[1].append(line)

    feed(path)
    return out


def _node_list(lines):
    ids = []
    for line in lines:
        for c in range(0, len(line), 10):
            s = line[c:c + 10].strip()
            if s:
                ids.append(int(s))
    return ids


class StarterDeck:
    """Content of a starter deck: the keywords listed in the module docstring."""

    def __init__(self, path):
        self.path = path
        self.title = ""
        self.invers = 0
        self.nodes = {}            # id -> (x, y, z), file order
        self.shells = {}           # part id -> list of (elem id, n1, n2, n3, n4)
        self.parts = {}            # id -> (prop id, mat id)
        self.props = {}            # id -> dict
        self.mats = {}             # id -> dict
        self.grnod = {}            # id -> list of node ids
        self.bcs = []              # (tra code, rot code, grnod id)
        self.inivel = []           # (vx, vy, vz, grnod id)
        self.admas = []            # (mass, grnod id)
        self.def_shell = dict(ishell=0, ismstr=0, ithick=0, iplas=0)
        self.def_solid = dict(isolid=0, ismstr=0, iframe=0)
        self.ishfram = 0
        self.bricks = {}           # part id -> list of (elem id, n1..n8)
        self.shell_thk = {}        # part id -> {elem id: thickness} of the /SHELL cards that give one
        self.funct = {}            # id -> (x list, y list)
        self.skews = {}            # id -> 9 floats (x', y', z')
        self.surf_seg = {}         # id -> list of (n1, n2, n3, n4), n4 = 0 for triangles
        self.surf_part = {}        # id -> list of part ids
        self.cload = []            # dict(func, dir, skew, grnod, ascale_x, fscale)
        self.grnod_grnod = {}      # id -> list of /GRNOD ids (resolved into grnod after reading)
        self.rbody = []            # dict per /RBODY card, deck order
        self.pload = []            # dict(surf, func, ascale_x, fscale)
        for key, lines, where in _blocks(path):
            self._block(key, lines, where)
        self._resolve_group_groups()

    def _resolve_group_groups(self):
        """/GRNOD/GRNOD: the union of its member groups' nodes, in /NODE order."""
        order = {n: k for k, n in enumerate(self.nodes)}
        pending = dict(self.grnod_grnod)
        while pending:
            done = [g for g, members in pending.items() if all(m in self.grnod for m in members)]
            if not done:
                raise RadError(f"/GRNOD/GRNOD {sorted(pending)}: undefined or cyclic member groups")
            for g in done:
                nodes = {n for m in pending.pop(g) for n in self.grnod[m]}
                self.grnod[g] = sorted(nodes, key=lambda n: order.get(n, n))

    def _block(self, key, L, where):
        k0 = key[0].upper()
        if k0 == "BEGIN":
            self.title = L[0].strip() if L else ""
            self.invers = _int(L[1], 0) if len(L) > 1 else 0
            if self.invers < 2017:
                raise RadError(f"{where}: input version {self.invers}: only the 2017+ block format is read")
        elif k0 in _IGNORED_STARTER:
            if k0 == "RANDOM" and L and _real(L[0], 0) != 0.0:
                raise RadError(f"{where}: /RANDOM noise is not implemented")
        elif k0 == "NODE":
            for line in L:
                self.nodes[_int(line, 0)] = (_real(line, 10), _real(line, 30), _real(line, 50))
        elif k0 == "SHELL":
            part = int(key[1])
            rows = self.shells.setdefault(part, [])
            thk = self.shell_thk.setdefault(part, {})
            for line in L:
                row = tuple(_int(line, 10 * c) for c in range(5))
                rows.append(row)
                t = _real(line, 80) if len(line) > 80 else 0.0
                if t > 0.0:
                    thk[row[0]] = t          # element thickness overriding the property's
        elif k0 == "BRICK":
            part = int(key[1])
            rows = self.bricks.setdefault(part, [])
            for line in L:
                rows.append(tuple(_int(line, 10 * c) for c in range(9)))
        elif k0 == "FUNCT":
            xs, ys = [], []
            for line in L[1:]:
                xs.append(_real(line, 0))
                ys.append(_real(line, 20))
            self.funct[int(key[1])] = (xs, ys)
        elif k0 == "SKEW":
            if key[1].upper() != "FIX":
                raise RadError(f"{where}: /SKEW/{key[1]} (moving frames) is not implemented")
            Y = np.array([_real(L[2], 20 * c) for c in range(3)])
            Z = np.array([_real(L[3], 20 * c) for c in range(3)])
            if Y[0] == 0.0 and Y[2] == 0.0:
                Y[1] = math.copysign(1.0, Y[1])
            if Z[0] == 0.0 and Z[1] == 0.0:
                Z[2] = math.copysign(1.0, Z[2])
            X = np.cross(Y, Z)
            Y = np.cross(Z, X)
            ax = [v / np.linalg.norm(v) for v in (X, Y, Z)]
            self.skews[int(key[2])] = np.concatenate(ax)
        elif k0 == "SURF":
            kind = key[1].upper()
            if kind == "SEG":
                self.surf_seg[int(key[2])] = [tuple(_int(line, 10 * c) for c in range(1, 5)) for line in L[1:]]
            elif kind == "PART":
                self.surf_part[int(key[2])] = _node_list(L[1:])
            else:
                raise RadError(f"{where}: /SURF/{key[1]} is not implemented")
        elif k0 == "CLOAD":
            line = L[1]
            if _int(line, 30) != 0:
                raise RadError(f"{where}: /CLOAD with a sensor is not implemented")
            if _int(line, 50) not in (0, 1):
                raise RadError(f"{where}: /CLOAD with a displacement or velocity abscissa is not implemented")
            dirs = {"X": 1, "Y": 2, "Z": 3, "XX": 4, "YY": 5, "ZZ": 6}
            d = line[10:20].strip().upper()
            if d not in dirs:
                raise RadError(f"{where}: /CLOAD direction {d!r}")
            self.cload.append(dict(func=_int(line, 0), dir=dirs[d], skew=_int(line, 20), grnod=_int(line, 40),
                                   ascale_x=_real(line, 60) or 1.0, fscale=_real(line, 80) or 1.0))
        elif k0 == "PLOAD":
            line = L[1]
            if _int(line, 20) != 0:
                raise RadError(f"{where}: /PLOAD with a sensor is not implemented")
            self.pload.append(dict(surf=_int(line, 0), func=_int(line, 10), ascale_x=_real(line, 60) or 1.0,
                                   fscale=_real(line, 80) or 1.0))
        elif k0 == "DEF_SOLID":
            if _int(L[0], 60) != 0:
                raise RadError(f"{where}: /DEF_SOLID Imas (nodal mass distribution) is not implemented")
            self.def_solid = dict(isolid=_int(L[0], 0), ismstr=_int(L[0], 10), iframe=_int(L[0], 70))
        elif k0 == "PART":
            self.parts[int(key[1])] = (_int(L[1], 0), _int(L[1], 10))
        elif k0 == "PROP" and key[1].upper() in ("SOLID", "TYPE14"):
            pid = int(key[2])
            if len(L) > 3 and _real(L[3], 0) != 0.0:
                raise RadError(f"{where}: /PROP/SOLID deltaT_min (small-strain switch) is not implemented")
            if _int(L[1], 20) != 0:
                raise RadError(f"{where}: /PROP/SOLID Iale is not on the element-cycle path")
            self.props[pid] = dict(kind="solid", isolid=_int(L[1], 0), ismstr=_int(L[1], 10), iframe=_int(L[1], 70),
                                   qa=_real(L[2], 0), qb=_real(L[2], 20), qh=_real(L[2], 40))
        elif k0 == "PROP":
            if key[1].upper() not in ("SHELL", "TYPE1"):
                raise RadError(f"{where}: /PROP/{key[1]} is not on the element-cycle path")
            pid = int(key[2])
            self.props[pid] = dict(kind="shell",
                ishell=_int(L[1], 0), ismstr=_int(L[1], 10), ish3n=_int(L[1], 20), idrill=_int(L[1], 30),
                hm=_real(L[2], 0), hf=_real(L[2], 20), hr=_real(L[2], 40), dm=_real(L[2], 60), dn=_real(L[2], 80),
                n=_int(L[3], 0), istrain=_int(L[3], 10), thick=_real(L[3], 20), ashear=_real(L[3], 40),
                ithick=_int(L[3], 60), iplas=_int(L[3], 70))
        elif k0 == "MAT":
            law = key[1].upper()
            mid = int(key[2])
            if law in ("PLAS_JOHNS", "LAW2"):
                if _int(L[2], 40) != 0:
                    raise RadError(f"{where}: /MAT/PLAS_JOHNS Iflag != 0 is not implemented")
                c = _real(L[4], 0) if len(L) > 4 else 0.0
                m = _real(L[5], 0) if len(L) > 5 else 0.0
                if c != 0.0 or m != 0.0:
                    raise RadError(f"{where}: strain-rate or thermal Johnson-Cook terms are not implemented")
                self.mats[mid] = dict(law=2, rho=_real(L[1], 0), E=_real(L[2], 0), nu=_real(L[2], 20),
                                      a=_real(L[3], 0), b=_real(L[3], 20), n=_real(L[3], 40),
                                      epsmax=_real(L[3], 60), sigmax=_real(L[3], 80))
            elif law in ("ELAST", "LAW1"):
                self.mats[mid] = dict(law=1, rho=_real(L[1], 0), E=_real(L[2], 0), nu=_real(L[2], 20))
            else:
                raise RadError(f"{where}: /MAT/{key[1]} is not on the element-cycle path")
        elif k0 == "DEF_SHELL":
            self.def_shell = dict(ishell=_int(L[0], 0), ismstr=_int(L[0], 10), ithick=_int(L[0], 20),
                                  iplas=_int(L[0], 30))
        elif k0 == "SHFRA":
            if len(key) < 2 or key[1].upper() != "V4":
                raise RadError(f"{where}: /SHFRA only as /SHFRA/V4")
            self.ishfram = 2           # contrl.F:478-486
        elif k0 == "BCS":
            line = L[1]
            tra, rot = line[3:6], line[7:10]
            code = lambda s: sum(b for ch, b in zip(s.replace(" ", "0"), (4, 2, 1)) if ch == "1")
            self.bcs.append((code(tra), code(rot), _int(line, 20), _int(line, 10)))
        elif k0 == "GRNOD":
            kind = key[1].upper()
            if kind == "NODE":
                self.grnod[int(key[2])] = _node_list(L[1:])
            elif kind == "GRNOD":
                self.grnod_grnod[int(key[2])] = _node_list(L[1:])
            else:
                raise RadError(f"{where}: /GRNOD/{key[1]} is not implemented")
        elif k0 == "RBODY":
            line = L[1]
            rb = dict(id=int(key[1]), master=_int(line, 0), isens=_int(line, 10), nskew=_int(line, 20),
                      ispher=_int(line, 30), mass=_real(line, 40), grnod=_int(line, 60), icog=_int(line, 80),
                      surf=_int(line, 90),
                      j=[_real(L[2], 20 * c) for c in range(3)] if len(L) > 2 else [0.0] * 3,
                      jc=[_real(L[3], 20 * c) for c in range(3)] if len(L) > 3 else [0.0] * 3,
                      ioptoff=_int(L[4], 0) if len(L) > 4 else 0, ifail=_int(L[4], 20) if len(L) > 4 else 0)
            if rb["isens"] or rb["nskew"] or rb["surf"] or rb["ioptoff"] or rb["ifail"]:
                raise RadError(f"{where}: /RBODY with a sensor, skew, surface, Ioptoff or Ifail is not implemented")
            if rb["icog"] not in (0, 1) or rb["ispher"] not in (0, 2):
                raise RadError(f"{where}: /RBODY ICoG {rb['icog']} / Ispher {rb['ispher']}; the element "
                               "cycle implements ICoG 1 and Ispher 2 (their defaults)")
            self.rbody.append(rb)
        elif k0 == "INIVEL":
            if key[1].upper() != "TRA":
                raise RadError(f"{where}: /INIVEL/{key[1]} is not implemented")
            line = L[1]
            if _int(line, 70) != 0:
                raise RadError(f"{where}: /INIVEL with a skew frame is not implemented")
            self.inivel.append((_real(line, 0), _real(line, 20), _real(line, 40), _int(line, 60)))
        elif k0 == "ADMAS":
            if int(key[1]) != 0:
                raise RadError(f"{where}: /ADMAS type {key[1]} is not implemented")
            self.admas.append((_real(L[1], 0), _int(L[1], 20)))
        else:
            raise RadError(f"{where}: keyword /{'/'.join(key)} is not implemented")


class EngineDeck:
    """Content of one engine deck: final time and rigid velocity links."""

    def __init__(self, path):
        self.path = path
        self.tstop = None
        self.rlinks = []            # dict(ic, icr, nodes=[ids])
        for key, lines, where in _blocks(path):
            k0 = key[0].upper()
            if k0 == "RUN":
                self.tstop = _real(lines[0], 0)
            elif k0 == "VEL":
                kind = key[1].upper()
                dirs = key[2].upper() if len(key) > 2 else "XYZ"
                if len(key) > 3 and int(key[3]) != 0:
                    raise RadError(f"{where}: /VEL with a skew frame is not implemented")
                if kind not in ("TRA", "ROT"):
                    raise RadError(f"{where}: /VEL/{key[1]} is not implemented")
                ic = sum(b for ch, b in (("X", 4), ("Y", 2), ("Z", 1)) if ch in dirs)
                self.rlinks.append(dict(ic=ic if kind == "TRA" else 0, icr=ic if kind == "ROT" else 0,
                                        nodes=_node_list(lines)))
            elif k0 in _IGNORED_ENGINE:
                pass
            else:
                raise RadError(f"{where}: engine keyword /{'/'.join(key)} is not implemented")
        if self.tstop is None:
            raise RadError(f"{path}: no /RUN card")


def _shell_flags(sd, prop):
    """Ishell, ISMSTR, ITHK and Iplas after the starter's defaults (the engine's
    IHBE follows from Ishell in the library, hm_read_prop01.F:305-315)."""
    ds = sd.def_shell
    ihbe = prop["ishell"] or ds["ishell"] or 1
    ismstr = prop["ismstr"] or ds["ismstr"] or 2
    ithk = prop["ithick"] or ds["ithick"]
    ipla = prop["iplas"] or ds["iplas"]
    return ihbe, ismstr, ithk, ipla


def _material(mat):
    if mat["law"] == 2:
        return decks.material(decks.LAW_JOHNSON_COOK, mat["rho"], mat["E"], mat["nu"], jc_a=mat["a"],
                              jc_b=mat["b"], jc_n=mat["n"],
                              epsmax=mat["epsmax"] if mat["epsmax"] > 0.0 else 1e20,
                              sigmax=mat["sigmax"] if mat["sigmax"] > 0.0 else 1e20)
    return decks.material(decks.LAW_ELASTIC, mat["rho"], mat["E"], mat["nu"])


def to_deck(sd: StarterDeck, name=None):
    """The element-cycle deck of a starter deck: one part with every node (in
    the order of /NODE); one hexa group per /PART with /BRICK elements, then one
    shell group per /PART with /SHELL elements, each in ascending part id; the
    time functions, skew frames, loads and skewed BCs; and ``ids`` (node ids) /
    ``hex_ids`` / ``elem_ids`` (element ids per hexa / shell group) for
    reporting."""
    ids = np.array(list(sd.nodes.keys()), np.int64)
    x = np.array(list(sd.nodes.values()), np.float64)
    index = {int(i): k for k, i in enumerate(ids)}
    part = decks.new_part(x)
    hex_ids, elem_ids = [], []
    for pid in sorted(sd.bricks):
        if pid not in sd.parts:
            raise RadError(f"/BRICK/{pid}: no /PART/{pid}")
        prop_id, mat_id = sd.parts[pid]
        prop, mat = sd.props[prop_id], sd.mats[mat_id]
        if prop.get("kind") != "solid":
            raise RadError(f"/PART/{pid}: bricks need a /PROP/SOLID")
        ds = sd.def_solid
        isolid = prop["isolid"] or ds["isolid"] or 1
        ismstr = prop["ismstr"] or ds["ismstr"] or 4
        iframe = prop["iframe"] or ds["iframe"] or 1
        if isolid != 1 or ismstr != 4 or iframe not in (1, 2):
            raise RadError(f"/PROP/SOLID/{prop_id}: Isolid {isolid} / Ismstr {ismstr} / Iframe {iframe}; the "
                           "element cycle implements Isolid 1 with Ismstr 4 and Iframe 1 or 2")
        rows = sorted(sd.bricks[pid])
        conn = np.array([[index[n] for n in r[1:]] for r in rows], np.int64)
        sp = decks.solid_prop(qa=prop["qa"] or 1.1, qb=prop["qb"] or 0.05, qh=prop["qh"] or 0.1,
                              jcvt=iframe - 1)              # IGEO(16) = Iframe - 1 (hm_read_prop14.F:380)
        decks.add_hex(part, conn, _material(mat), sp)
        hex_ids.append(np.array([r[0] for r in rows], np.int64))
    for pid in sorted(sd.shells):
        if pid not in sd.parts:
            raise RadError(f"/SHELL/{pid}: no /PART/{pid}")
        prop_id, mat_id = sd.parts[pid]
        prop, mat = sd.props[prop_id], sd.mats[mat_id]
        if prop.get("kind") != "shell":
            raise RadError(f"/PART/{pid}: shells need a /PROP/SHELL")
        ihbe, ismstr, ithk, ipla = _shell_flags(sd, prop)
        if ithk == 2:
            ithk = 0                        # cgrtails.F:832-833
        if ihbe not in (1, 2, 3, 4) or ismstr != 2:
            raise RadError(f"/PROP/SHELL/{prop_id}: Ishell {ihbe} / Ismstr {ismstr}; the element cycle "
                           "implements Ishell 1 to 4 with Ismstr 2")
        if ipla not in (0, 1, 2, 3):
            raise RadError(f"/PROP/SHELL/{prop_id}: Iplas {ipla}")
        # M2CPLR's IPLA from Iplas (cgrtails.F:822-829; the explicit default Iplas 0
        # stays 0): 0 and 2 radial return, 1 Newton iterations, 3 normal projection
        ipla = {0: 0, 1: 1, 2: 0, 3: 2}[ipla]
        if prop["dm"] != 0.0:
            raise RadError(f"/PROP/SHELL/{prop_id}: membrane damping dm is not implemented")
        npt = prop["n"]
        if npt == 0:
            if mat["law"] == 2:
                npt = 3                     # cgrtails.F:795-806
            else:
                raise RadError(f"/PROP/SHELL/{prop_id}: global integration (N = 0) with LAW1")
        if not 1 <= npt <= 10:
            raise RadError(f"/PROP/SHELL/{prop_id}: N = {npt}")
        rows = sorted(sd.shells[pid])
        conn = np.array([[index[n] for n in r[1:]] for r in rows], np.int64)
        # hourglass defaults: 0.1 / 0.1 / 0.01 for Ishell 3, 0.01 otherwise
        # (hm_read_prop01.F:204-212)
        hdef = (0.1, 0.1, 0.01) if ihbe == 3 else (0.01, 0.01, 0.01)
        p = decks.shell_prop(prop["thick"], npt=npt, ithk=1 if ithk > 0 else 0,
                             hm=prop["hm"] or hdef[0], hf=prop["hf"] or hdef[1], hr=prop["hr"] or hdef[2],
                             ishfram=sd.ishfram, ishell=ihbe, dn=prop["dn"])
        p["ipla"] = ipla
        if prop["ashear"] != 0.0:
            p["shf"] = prop["ashear"]
        if npt == 1:
            p["shf"] = 0.0
        et = sd.shell_thk.get(pid, {})
        thke = np.array([et.get(r[0], prop["thick"]) for r in rows], np.float64) if et else None
        decks.add_shell(part, conn, _material(mat), p, thke=thke)
        elem_ids.append(np.array([r[0] for r in rows], np.int64))
    skew_index = {sid: k for k, sid in enumerate(sorted(sd.skews))}
    skew_of = lambda sid, what: -1 if sid == 0 else _lookup(skew_index, sid, what)
    iskew = -np.ones(x.shape[0], np.int32)
    for tra, rot, g, sk in sd.bcs:
        for n in sd.grnod[g]:
            part["icodt"][index[n]] |= tra
            part["icodr"][index[n]] |= rot
            if sk:
                iskew[index[n]] = skew_of(sk, "/BCS skew")
    if (iskew >= 0).any():
        part["iskew"] = iskew
    for vx, vy, vz, g in sd.inivel:
        for n in sd.grnod[g]:
            part["v"][index[n]] = (vx, vy, vz)
    for mass, g in sd.admas:
        for n in sd.grnod[g]:
            part["ms"][index[n]] += mass
    if sd.rbody:
        part["rbodies"] = []
        for rb in sd.rbody:
            if rb["grnod"] not in sd.grnod:
                raise RadError(f"/RBODY/{rb['id']}: node group {rb['grnod']} is not defined")
            m = index[rb["master"]]
            slaves = [index[n] for n in sd.grnod[rb["grnod"]] if index[n] != m]
            rby, tensor = rbody_init(part, m, slaves, rb["mass"], rb["j"], rb["jc"])
            part["rbodies"].append(dict(id=rb["id"], master=m, slaves=np.array(slaves, np.int64), rby=rby,
                                        tensor=tensor))
    func_index = {fid: k for k, fid in enumerate(sorted(sd.funct))}
    cloads, ploads = [], []
    for c in sd.cload:
        cloads.append(dict(nodes=np.array([index[n] for n in sd.grnod[c["grnod"]]], np.int64), dir=c["dir"],
                           skew=skew_of(c["skew"], "/CLOAD skew"), func=_lookup(func_index, c["func"], "/CLOAD"),
                           ascale_x=c["ascale_x"], fscale=c["fscale"]))
    for q in sd.pload:
        seg = _segments(sd, q["surf"], index)
        ploads.append(dict(seg=seg, func=_lookup(func_index, q["func"], "/PLOAD"), ascale_x=q["ascale_x"],
                           fscale=q["fscale"]))
    if cloads:
        part["cloads"] = cloads
    if ploads:
        part["ploads"] = ploads
    part["ids"] = ids
    part["hex_ids"] = hex_ids
    part["elem_ids"] = elem_ids
    d = decks.deck([part], name=name or sd.title or "rad")
    if sd.funct:
        d["functions"] = [dict(x=sd.funct[f][0], y=sd.funct[f][1]) for f in sorted(sd.funct)]
    if sd.skews:
        d["skews"] = [sd.skews[k] for k in sorted(sd.skews)]
    return d


def principal_inertia(I):
    """Eigenvalues and unit eigenvectors (columns) of a symmetric 3x3 inertia
    tensor by cyclic Jacobi rotations, the eigenvalues left in the positions of
    the diagonal they come from (a diagonal tensor is returned as it is); the
    principal frame of INEPRI / VALPR (inepri.F)."""
    a = np.array(I, np.float64)
    v = np.eye(3)
    for _ in range(50):
        off = abs(a[0, 1]) + abs(a[0, 2]) + abs(a[1, 2])
        if off <= 1e-30 * (abs(a[0, 0]) + abs(a[1, 1]) + abs(a[2, 2])) or off == 0.0:
            break
        for p, q in ((0, 1), (0, 2), (1, 2)):
            if a[p, q] == 0.0:
                continue
            theta = (a[q, q] - a[p, p]) / (2.0 * a[p, q])
            t = math.copysign(1.0, theta) / (abs(theta) + math.sqrt(theta * theta + 1.0))
            c = 1.0 / math.sqrt(t * t + 1.0)
            s_ = t * c
            rot = np.eye(3)
            rot[p, p] = rot[q, q] = c
            rot[p, q], rot[q, p] = s_, -s_
            a = rot.T @ a @ rot
            v = v @ rot
    return np.diag(a).copy(), v


def rbody_init(part, m, slaves, mass, j, jc):
    """Starter initialisation of a rigid body (INIRBY, inirby.F:146-330, 340-361,
    715-836; 3D, no skew, ICoG 1, Ispher 2): the main node takes the added mass
    and inertia, moves to the centre of mass of itself and the secondary nodes,
    and gets the body's mass; the inertia tensor about the new position is
    assembled from the main node's own mass and inertia and every secondary
    node's; its principal frame and inertias are returned as 12 values (the three
    unit axes, then the three inertias, as RBY(1:12)) with the inertia tensor
    itself; the main node's rotational inertia becomes the smallest principal
    inertia.  part's ms, inr and x are updated in place."""
    ms, inr, x = part["ms"], part["inr"], part["x"]
    ms[m] += mass
    if ms[m] == 0.0:
        ms[m] = 1e-20
    jxx, jyy, jzz = j
    jxy, jyz, jxz = jc
    I = np.array([[jxx, jxy, jxz], [jxy, jyy, jyz], [jxz, jyz, jzz]], np.float64)
    for c in range(3):
        I[c, c] += inr[m]
    xmg = ms[m]
    xg = x[m].copy()
    acc = x[m] * ms[m]
    masrb = ms[m]
    for n in slaves:
        acc = acc + x[n] * ms[n]
        masrb += ms[n]
    x[m] = acc / masrb
    d = xg - x[m]
    I[0, 0] += (d[1] * d[1] + d[2] * d[2]) * xmg
    I[0, 1] -= d[0] * d[1] * xmg
    I[0, 2] -= d[0] * d[2] * xmg
    I[1, 0] -= d[0] * d[1] * xmg
    I[1, 1] += (d[2] * d[2] + d[0] * d[0]) * xmg
    I[1, 2] -= d[1] * d[2] * xmg
    I[2, 0] -= d[0] * d[2] * xmg
    I[2, 1] -= d[1] * d[2] * xmg
    I[2, 2] += (d[0] * d[0] + d[1] * d[1]) * xmg
    if len(slaves) == 1:
        for c in range(3):
            I[c, c] += 1e-20
    for n in slaves:
        r = x[n] - x[m]
        xx, xy, xz, yy, yz, zz = r[0] * r[0], r[0] * r[1], r[0] * r[2], r[1] * r[1], r[1] * r[2], r[2] * r[2]
        I[0, 0] += inr[n] + (yy + zz) * ms[n]
        I[0, 1] -= xy * ms[n]
        I[0, 2] -= xz * ms[n]
        I[1, 0] -= xy * ms[n]
        I[1, 1] += inr[n] + (zz + xx) * ms[n]
        I[1, 2] -= yz * ms[n]
        I[2, 0] -= xz * ms[n]
        I[2, 1] -= yz * ms[n]
        I[2, 2] += inr[n] + (xx + yy) * ms[n]
    ip, axes = principal_inertia(I)
    imin, imax = ip.min(), ip.max()
    if imin <= 1e-3 * imax:                       # Ispher 2 (inirby.F:744-751)
        ip = np.where(ip / imax < 1e-3, ip + 0.1 * imax, ip)
    ms[m] = masrb
    inr[m] = ip.min()
    return np.concatenate([axes[:, 0], axes[:, 1], axes[:, 2], ip]), I


def _lookup(table, key, what):
    if key not in table:
        raise RadError(f"{what}: id {key} is not defined")
    return table[key]


def _segments(sd, surf, index):
    """0-based segments (nseg, 4) of a surface, -1 in the fourth column of a
    three-node segment."""
    if surf in sd.surf_seg:
        rows = [[index[n] for n in r[:3]] + [index[r[3]] if r[3] else -1] for r in sd.surf_seg[surf]]
    elif surf in sd.surf_part:
        rows = []
        for pid in sd.surf_part[surf]:
            if pid in sd.bricks:
                raise RadError(f"/SURF/PART/{surf}: faces of solid parts are not implemented")
            rows += [[index[n] for n in r[1:5]] for r in sorted(sd.shells.get(pid, []))]
    else:
        raise RadError(f"/PLOAD: surface {surf} is not defined")
    return np.array(rows, np.int64).reshape(-1, 4)


def add_engine(deck, ed: EngineDeck):
    """The rigid links of an engine deck, as ``rlinks`` of the deck's part
    (node ids mapped to 0-based node indices)."""
    part = deck["parts"][0]
    index = {int(i): k for k, i in enumerate(part["ids"])}
    part["rlinks"] = [dict(ic=r["ic"], icr=r["icr"], nodes=np.array([index[n] for n in r["nodes"]], np.int64))
                      for r in ed.rlinks]
    return deck


def element_id(deck, ityptst, neltst):
    """User id of the element that set the time step (ityptst 1: hexa, 3: shell)."""
    if neltst < 0 or ityptst not in (1, 3):
        return None
    for ids in deck["parts"][0]["hex_ids" if ityptst == 1 else "elem_ids"]:
        if neltst < ids.size:
            return int(ids[neltst])
        neltst -= ids.size
    return None


def part_masses(deck):
    """Structural mass of each shell group (rho t A), as the starter's
    PART MASS table prints it."""
    part = deck["parts"][0]
    out = []
    for g in part["shell"]:
        conn = g["ixc"][:, 1:5] - 1
        area = decks.shell_areas(part["x"], conn)
        out.append(float(np.sum(g["mat"]["rho0"] * g["thke"] * area)))
    return out


def total_mass(deck):
    return float(np.sum(deck["parts"][0]["ms"]))


# ---------------------------------------------------------------------------
# writer: a deck dict as a starter deck and an engine deck (2019 block format)
# ---------------------------------------------------------------------------

def _num20(x):
    """A real in at most 19 characters, so that a blank separates the fields: the
    shortest exact form when it fits, else 13 significant digits (a 20-character
    field cannot hold every double)."""
    r = repr(float(x))
    return r if len(r) <= 19 else f"{float(x):.13g}"


def _f20(*v):
    return "".join(f"{_num20(x):>20s}" for x in v)


def _i10(*v):
    return "".join(f"{int(x):10d}" for x in v)


def _grnod(L, gid, title, nodes):
    L += [f"/GRNOD/NODE/{gid}", title]
    nodes = [int(n) for n in nodes]
    L += [_i10(*nodes[i:i + 10]) for i in range(0, len(nodes), 10)]


def write_starter(deck, path, part=0, title=None):
    """Writes part ``part`` of a deck dict as a Radioss starter deck: /NODE,
    /BRICK and /SHELL per element group (one /PART, /PROP and /MAT each),
    /BCS, /INIVEL/TRA and /ADMAS from the nodal arrays (the added mass is the
    nodal mass beyond the lumped element masses), /SKEW/FIX, /FUNCT, /CLOAD and
    /PLOAD; a shell group's uniform ``pressure`` becomes a /PLOAD with a
    constant function.  Node and element ids are 1-based indices.  Per-element
    yield stresses have no deck form and are refused."""
    p = deck["parts"][part]
    x = p["x"]
    n = x.shape[0]
    L = ["#RADIOSS STARTER", "/BEGIN", title or deck.get("name", "deck"), _i10(2019, 0),
         f"{'kg':>20s}{'m':>20s}{'s':>20s}", f"{'kg':>20s}{'m':>20s}{'s':>20s}",
         "/TITLE", title or deck.get("name", "deck"), "/NODE"]
    L += [_i10(k + 1) + _f20(*x[k]) for k in range(n)]
    mass = np.zeros(n)
    pid = 0
    eid = 0
    gid = 0
    fid_const = None
    funcs = list(deck.get("functions", []))
    ploads = list(p.get("ploads", []))
    for g in p["hex"]:
        pid += 1
        m = g["mat"]
        conn = g["ixs"][:, 1:9] - 1
        vol0 = np.asarray(g["vol0"]) if g.get("vol0") is not None else decks.hex_volumes(x, conn)
        np.add.at(mass, conn.ravel(), np.repeat(m["rho0"] * vol0 / 8.0, 8))
        L += _material_cards(pid, m)
        pr = g["prop"]
        L += [f"/PROP/SOLID/{pid}", f"solid {pid}", _i10(1, 4, 0, 0, 0, 0, 0, 1 + pr.get("jcvt", 0)) + _f20(0.0),
              _f20(pr["qa"], pr["qb"], pr["qh"], 0.0, 0.0), _f20(0.0, 0.0, 0.0, 0.0, 0.0),
              f"/PART/{pid}", f"part {pid}", _i10(pid, pid, 0), f"/BRICK/{pid}"]
        for e in range(conn.shape[0]):
            eid += 1
            L.append(_i10(eid, *(conn[e] + 1)))
    for g in p["shell"]:
        pid += 1
        m, pr = g["mat"], g["prop"]
        if g.get("jc_a") is not None:
            raise ValueError("write_starter: per-element yield stresses have no .rad form")
        conn = g["ixc"][:, 1:5] - 1
        thk = np.asarray(g["thke"], np.float64)
        area = decks.shell_areas(x, conn)
        ems = m["rho0"] * thk * area / 4.0
        np.add.at(mass, conn.ravel(), np.repeat(ems, 4))
        L += _material_cards(pid, m)
        L += [f"/PROP/SHELL/{pid}", f"shell {pid}", _i10(int(pr.get("ishell", 1)) or 1, 2, 0, 0) + " " * 20 + _f20(0.0),
              _f20(pr["hm"], pr["hf"], pr["hr"], 0.0, float(pr.get("dn", 0.0))),
              _i10(pr["npt"], 0) + _f20(pr["thk"], pr["shf"] if pr["npt"] > 1 else 0.0) +
              _i10(1 if pr["ithk"] else 2, {0: 2, 1: 1, 2: 3}[int(pr.get("ipla", 0))]),
              f"/PART/{pid}", f"part {pid}", _i10(pid, pid, 0), f"/SHELL/{pid}"]
        uniform = np.allclose(thk, pr["thk"], rtol=0, atol=0)
        for e in range(conn.shape[0]):
            eid += 1
            L.append(_i10(eid, *(conn[e] + 1)) + ("" if uniform else " " * 10 + _f20(0.0, thk[e])))
        if pr.get("pressure", 0.0) != 0.0:
            if fid_const is None:
                funcs.append(dict(x=[0.0], y=[1.0]))
                fid_const = len(funcs) - 1
            ploads.append(dict(seg=conn, func=fid_const, ascale_x=1.0, fscale=-pr["pressure"]))
    if any(g["prop"].get("ishfram", 0) == 2 for g in p["shell"]):
        L.insert(L.index("/NODE"), "/SHFRA/V4")
    skews = deck.get("skews", [])
    for k, ax in enumerate(skews):
        ax = np.asarray(ax, np.float64).reshape(3, 3)
        L += [f"/SKEW/FIX/{k + 1}", f"skew {k + 1}", _f20(0.0, 0.0, 0.0), _f20(*ax[1]), _f20(*ax[2])]
    iskew = p.get("iskew")
    combos = {}
    for i in range(n):
        ct, cr = int(p["icodt"][i]), int(p["icodr"][i])
        if ct or cr:
            sk = int(iskew[i]) + 1 if iskew is not None and iskew[i] >= 0 else 0
            combos.setdefault((ct, cr, sk), []).append(i + 1)
    digits = lambda c: "".join("1" if c & b else "0" for b in (4, 2, 1))
    for k, ((ct, cr, sk), nodes) in enumerate(sorted(combos.items())):
        gid += 1
        L += [f"/BCS/{k + 1}", f"bcs {k + 1}", f"   {digits(ct)} {digits(cr)}" + _i10(sk, gid)]
        _grnod(L, gid, f"bcs {k + 1}", nodes)
    vels = {}
    for i in range(n):
        v = tuple(float(c) for c in p["v"][i])
        if any(v):
            vels.setdefault(v, []).append(i + 1)
    if np.abs(p["vr"]).max() > 0:
        raise ValueError("write_starter: initial rotational velocities are not written")
    for k, (v, nodes) in enumerate(sorted(vels.items())):
        gid += 1
        L += [f"/INIVEL/TRA/{k + 1}", f"inivel {k + 1}", _f20(*v) + _i10(gid, 0)]
        _grnod(L, gid, f"inivel {k + 1}", nodes)
    extra = np.asarray(p["ms"]) - mass
    added = np.nonzero(extra > 1e-12 * max(np.abs(p["ms"]).max(), 1e-300))[0]
    for k, i in enumerate(added):
        gid += 1
        L += [f"/ADMAS/0/{k + 1}", f"added mass {k + 1}", _f20(extra[i]) + _i10(gid)]
        _grnod(L, gid, f"added mass {k + 1}", [i + 1])
    for k, f in enumerate(funcs):
        L += [f"/FUNCT/{k + 1}", f"function {k + 1}"] + [_f20(a, b) for a, b in zip(f["x"], f["y"])]
    dname = {1: "X", 2: "Y", 3: "Z", 4: "XX", 5: "YY", 6: "ZZ"}
    for k, c in enumerate(p.get("cloads", [])):
        gid += 1
        sk = int(c.get("skew", -1)) + 1
        L += [f"/CLOAD/{k + 1}", f"cload {k + 1}",
              _i10(c["func"] + 1) + f"{dname[c['dir']]:>10s}" + _i10(sk, 0, gid, 1) +
              _f20(c.get("ascale_x", 1.0), c.get("fscale", 1.0))]
        _grnod(L, gid, f"cload {k + 1}", np.asarray(c["nodes"]) + 1)
    for k, q in enumerate(ploads):
        seg = np.asarray(q["seg"])
        L += [f"/SURF/SEG/{k + 1}", f"segments {k + 1}"]
        L += [_i10(j + 1, *[s + 1 if s >= 0 else 0 for s in seg[j]]) for j in range(seg.shape[0])]
        L += [f"/PLOAD/{k + 1}", f"pload {k + 1}",
              _i10(k + 1, q["func"] + 1, 0, 0) + " " * 20 + _f20(q.get("ascale_x", 1.0), q.get("fscale", 1.0))]
    L.append("/END")
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def _material_cards(mid, m):
    if m["law"] == decks.LAW_JOHNSON_COOK:
        return [f"/MAT/PLAS_JOHNS/{mid}", f"material {mid}", _f20(m["rho0"]), _f20(m["young"], m["nu"]) + _i10(0),
                _f20(m["jc_a"], m["jc_b"], m["jc_n"], 0.0 if m["epsmax"] >= 1e20 else m["epsmax"],
                     0.0 if m["sigmax"] >= 1e20 else m["sigmax"]),
                _f20(0.0, 0.0) + _i10(0, 0) + _f20(0.0, 0.0), _f20(0.0, 0.0, 0.0, 0.0)]
    return [f"/MAT/ELAST/{mid}", f"material {mid}", _f20(m["rho0"]), _f20(m["young"], m["nu"])]


def write_engine(path, run_name, tstop, deck=None, part=0, run=1):
    """Writes an engine deck: /RUN to ``tstop`` and the part's rigid links as /VEL cards."""
    L = ["#RADIOSS ENGINE", f"/RUN/{run_name}/{run}", _f20(tstop), "/PRINT/-100/55", "/PARITH/ON"]
    if deck is not None:
        for r in deck["parts"][part].get("rlinks", []):
            for kind, code in (("TRA", r.get("ic", 7)), ("ROT", r.get("icr", 0))):
                if code:
                    dirs = "".join(c for c, b in (("X", 4), ("Y", 2), ("Z", 1)) if code & b)
                    nodes = [int(v) + 1 for v in r["nodes"]]
                    L.append(f"/VEL/{kind}/{dirs}")
                    L += [_i10(*nodes[i:i + 10]) for i in range(0, len(nodes), 10)]
    L.append("/END")
    with open(path, "w") as f:
        f.write("\n".join(L) + "\n")


def _dt_estimate(deck, part=0):
    """Initial element time step, roughly: DTFAC * length / wave speed of the
    stiffest, smallest element (for the /RUN time of a written deck)."""
    p = deck["parts"][part]
    dt = np.inf
    for g in p["hex"]:
        m = g["mat"]
        conn = g["ixs"][:, 1:9] - 1
        vol = np.abs(decks.hex_volumes(p["x"], conn))
        c = np.sqrt((m["bulk"] + 4.0 / 3.0 * m["shear"]) / m["rho0"])
        dt = min(dt, deck.get("dtfac_solid", 0.9) * vol.min() ** (1.0 / 3.0) / c)
    for g in p["shell"]:
        conn = g["ixc"][:, 1:5] - 1
        dt = min(dt, deck.get("dtfac_shell", 0.9) * np.sqrt(decks.shell_areas(p["x"], conn).min()) /
                 g["mat"]["ssp_shell"])
    return dt


def main(argv=None):
    """Writes a workload as <NAME>_0000.rad (starter) and <NAME>_0001.rad (engine):

        python -m openradioss_b200.rad --workload hex_block --out DIR [--tstop T]
    """
    import argparse
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--workload", required=True, choices=["hex_block", "shell_plate", "mixed_mesh", "hat_rail"])
    ap.add_argument("--out", required=True)
    ap.add_argument("--name", default=None)
    ap.add_argument("--tstop", type=float, default=0.0, help="final time (default: cycles x initial dt estimate)")
    a = ap.parse_args(argv)
    make = {"hex_block": decks.c1_hex_block, "shell_plate": decks.c2_shell_plate, "mixed_mesh": decks.c4_mixed_mesh,
            "hat_rail": decks.hat_rail}[a.workload]
    d = make()
    name = (a.name or a.workload.upper().replace("_", ""))[:8]
    os.makedirs(a.out, exist_ok=True)
    tstop = a.tstop or d.get("ncycles", 100) * _dt_estimate(d)
    write_starter(d, os.path.join(a.out, f"{name}_0000.rad"))
    write_engine(os.path.join(a.out, f"{name}_0001.rad"), name, tstop, d)
    print(f"{a.out}/{name}_0000.rad, {name}_0001.rad (final time {tstop:.6g})")


if __name__ == "__main__":
    main()
