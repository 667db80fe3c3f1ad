"""The .rad writer: the synthetic workloads written as starter and engine decks
and read back must give the same deck (masses, inertias, codes, properties,
materials, loads, links) and run bitwise alike on the oracle.  This is how the
workloads reach the reference engine wherever it can be built."""
import numpy as np
import pytest

from openradioss_b200 import decks, rad


def roundtrip(deck, tmp_path, part=0):
    s = tmp_path / "RT_0000.rad"
    e = tmp_path / "RT_0001.rad"
    rad.write_starter(deck, str(s), part=part)
    rad.write_engine(str(e), "RT", 1e-3, deck, part=part)
    got = rad.add_engine(rad.to_deck(rad.StarterDeck(str(s))), rad.EngineDeck(str(e)))
    return got


def same_run(a, b, ncycles=40, tol=0.0):
    """Bitwise (tol 0) when every number of the deck fits a 20-character field
    exactly; otherwise within tol (a field holds 13 significant digits)."""
    from oracle.oracle import Oracle
    oa, ob = Oracle(a), Oracle(b)
    oa.step(ncycles)
    ob.step(ncycles)
    na, nb = oa.get_nodes(), ob.get_nodes()
    for k in ("x", "d", "v", "vr"):
        s = max(np.abs(na[k]).max(), 1e-300)
        assert np.abs(na[k] - nb[k]).max() <= tol * s, (k, np.abs(na[k] - nb[k]).max() / s)
    ea, eb = oa.energies(), ob.energies()
    for k in ea:
        assert abs(ea[k] - eb[k]) <= tol * max(abs(ea[k]), 1e-300), k


def test_hex_block_roundtrip(tmp_path):
    d = decks.c1_hex_block(nx=4, ny=4, nz=8, ncycles=40)
    got = roundtrip(d, tmp_path)
    pw, pg = d["parts"][0], got["parts"][0]
    assert np.allclose(pg["ms"], pw["ms"], rtol=1e-13, atol=0)
    assert (pg["icodt"] == pw["icodt"]).all() and np.array_equal(pg["v"], pw["v"])
    same_run(d, got)


def test_shell_plate_with_pressure_and_thickness_roundtrip(tmp_path):
    d = decks.c2_shell_plate(n=12, size=0.012, ncycles=40)
    d["parts"][0]["shell"][0]["thke"] = np.linspace(0.9e-3, 1.1e-3, 144)
    p = d["parts"][0]
    decks_ms = p["ms"].copy()
    p["ms"][:] = 0.0
    p["inr"][:] = 0.0
    g = p["shell"].pop()
    decks.add_shell(p, g["ixc"][:, 1:5] - 1, g["mat"], g["prop"], thke=g["thke"])
    assert not np.array_equal(decks_ms, p["ms"])
    got = roundtrip(d, tmp_path)
    pg = got["parts"][0]
    # jittered coordinates and linspace thicknesses do not fit a field exactly: 13 digits
    assert np.allclose(pg["ms"], p["ms"], rtol=1e-11, atol=0)
    assert np.allclose(pg["inr"], p["inr"], rtol=1e-11, atol=0)
    assert len(pg["ploads"]) == 1 and pg["ploads"][0]["fscale"] == -2e6
    # the group pressure becomes a /PLOAD: same forces, a load slot instead of the shell's own
    from oracle.oracle import Oracle
    oa, ob = Oracle(d), Oracle(got)
    oa.step(40)
    ob.step(40)
    assert np.abs(oa.get_nodes()["d"] - ob.get_nodes()["d"]).max() <= 1e-10 * np.abs(oa.get_nodes()["d"]).max()


def test_rail_with_link_and_loads_roundtrip(tmp_path):
    d = decks.hat_rail(length=0.1, kink=(0.03, 0.06))
    p = d["parts"][0]
    p["cloads"] = [dict(nodes=np.array([5, 9]), dir=2, skew=0, func=0, fscale=3.0)]
    d["functions"] = [dict(x=[0.0, 1e-4], y=[0.0, 1.0])]
    d["skews"] = [np.eye(3).reshape(9)]
    got = roundtrip(d, tmp_path)
    pg = got["parts"][0]
    assert np.allclose(pg["ms"], p["ms"], rtol=1e-13, atol=0)           # the added mass came back
    assert len(pg["rlinks"]) == 1 and (pg["rlinks"][0]["nodes"] == p["rlinks"][0]["nodes"]).all()
    assert pg["shell"][0]["prop"]["ishfram"] == 2
    same_run(d, got, tol=1e-10)        # linspace coordinates: 13 digits in the deck


def test_per_element_yield_is_refused(tmp_path):
    d = decks.c5_adjoint_plate(n=4, ncycles=5)
    with pytest.raises(ValueError):
        rad.write_starter(d, str(tmp_path / "X_0000.rad"))


def test_convected_frame_hexa_roundtrip(tmp_path):
    d = decks.c1_hex_block(nx=3, ny=3, nz=6, ncycles=40)
    d["parts"][0]["hex"][0]["prop"]["jcvt"] = 1         # /PROP/SOLID Iframe 2
    got = roundtrip(d, tmp_path)
    assert got["parts"][0]["hex"][0]["prop"]["jcvt"] == 1
    same_run(d, got)
