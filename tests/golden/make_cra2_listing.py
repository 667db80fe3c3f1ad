"""Extracts the golden values of the reference's miniqa RESTART/cra2 test
into cra2_listing.json (run from the repository root, next to a reference
checkout, whose location OR_REFERENCE_ROOT gives):

    OR_REFERENCE_ROOT=<reference checkout> python tests/golden/make_cra2_listing.py

From the reference engine's own listings (qa-tests/miniqa/RESTART/cra2/
reference/CRA2V44_0001.out and CRA2V44_0002.out) it takes every cycle line:
CYCLE, TIME, TIME-STEP, ELEMENT, I-ENERGY, K-ENERGY T, K-ENERGY R (each
printed with 4 significant digits); from the starter listing
(CRA2V44_0000.out) the PART MASS table and the total mass; and the values of
data/ref.extract (cycle 1800 of the second engine run).  The numbers are kept
as printed (strings) so that a test can compare at the printed precision.
"""
import json
import os
import re

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cra2_listing.json")

LINE = re.compile(r"^\s*(\d+)\s+(\S+)\s+(\S+)\s+SHELL\s+(\d+)\s+(\S+)%\s+(\S+)\s+(\S+)\s+(\S+)\s+")


def engine_lines(path):
    rows = []
    with open(path) as f:
        for line in f:
            m = LINE.match(line)
            if m:
                cyc, tt, dt, el, _err, ie, ke, ker = m.groups()
                rows.append(dict(cycle=int(cyc), time=tt, dt=dt, element=int(el), ie=ie, ke=ke, ker=ker))
            m = re.search(r"TOTAL NUMBER OF CYCLES\s*:\s*(\d+)", line)
            if m:
                ncyc = int(m.group(1))
    return rows, ncyc


def starter_masses(path):
    text = open(path).read()
    parts = [float(m.group(1)) for m in re.finditer(r"Mass\s+Ixx.*\n\s*(\S+)", text)]
    total = float(re.search(r"TOTAL MASS AND MASS CENTER.*?\n.*?\n\s+MASS.*\n\s*(\S+)", text).group(1))
    return parts, total


def extract(path):
    out = {}
    for line in open(path):
        f = line.split()
        if len(f) >= 3 and f[1] in ("CYCLE", "TIME", "TSTEP", "IENERGY", "KENERGYT", "KENERGYR"):
            out[f[1]] = f[2]
    return out


def main():
    ref = os.environ.get("OR_REFERENCE_ROOT")
    if not ref:
        raise SystemExit("set OR_REFERENCE_ROOT to a reference checkout")
    CASE = os.path.join(ref, "qa-tests", "miniqa", "RESTART", "cra2")
    r1, n1 = engine_lines(os.path.join(CASE, "reference", "CRA2V44_0001.out"))
    r2, n2 = engine_lines(os.path.join(CASE, "reference", "CRA2V44_0002.out"))
    parts, total = starter_masses(os.path.join(CASE, "reference", "CRA2V44_0000.out"))
    data = dict(source="qa-tests/miniqa/RESTART/cra2 (reference listings, OpenRadioss engine)",
                part_mass=parts, total_mass=total,
                runs=[dict(tstop=2.5, rigid_link=True, total_cycles=n1, lines=r1),
                      dict(tstop=5.0, rigid_link=False, total_cycles=n2, lines=r2)],
                ref_extract=extract(os.path.join(CASE, "data", "ref.extract")))
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)
    print(f"{OUT}: {len(r1)} + {len(r2)} cycle lines")


if __name__ == "__main__":
    main()
