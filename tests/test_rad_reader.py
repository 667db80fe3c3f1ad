"""The .rad reader on a deck written here in the reference's 2019 block format
(card layouts of hm_cfg_files radioss2019+): a LAW1 hexa block under a /PLOAD
on /SURF/SEG segments and a /CLOAD in a /SKEW/FIX frame, held at its base by a
skewed /BCS, next to a LAW2 shell strip loaded by a /PLOAD on /SURF/PART.

The deck the reader builds must equal the one built directly with
openradioss_b200.decks (same masses, codes, loads, functions and frames),
and both must run identically on the oracle.  Unknown or unsupported keywords
must be refused.
"""
import numpy as np
import pytest

from openradioss_b200 import decks, rad

E, NU, RHO = 210e3, 0.3, 7.85e-9        # N, mm, t, s


def f20(*v):
    return "".join(f"{x:20.10g}" for x in v)


def i10(*v):
    return "".join(f"{int(x):10d}" for x in v)


def write_deck(path):
    xb, cb = decks.hex_block(2, 2, 3, 1.0)
    xs, cs, _ = decks.quad_plate(3, 3.0)
    xs = xs + [5.0, 0.0, 0.0]
    x = np.vstack([xb, xs])
    cs = cs + xb.shape[0]
    L = ["#RADIOSS STARTER", "/BEGIN", "reader test", i10(2019, 0), f20(1, 1, 1), f20(1, 1, 1),
         "/NODE"]
    L += [i10(k + 1) + f20(*x[k]) for k in range(x.shape[0])]
    L += ["/MAT/ELAST/1", "steel", f20(RHO), f20(E, NU),
          "/MAT/PLAS_JOHNS/2", "steel", f20(RHO), f20(E, NU) + i10(0), f20(350.0, 275.0, 0.36, 0.0, 0.0),
          f20(0.0, 0.0) + i10(0, 0) + f20(0.0, 0.0), f20(0.0, 0.0, 0.0, 0.0),
          "/PROP/SOLID/1", "solid", i10(0, 0, 0, 0, 0, 0, 0, 0) + f20(0.0), f20(0.0, 0.0, 0.0, 0.0, 0.0),
          f20(0.0, 0.0, 0.0, 0.0, 0.0),
          "/PROP/SHELL/2", "shell", i10(0, 0, 0, 0) + " " * 20 + f20(0.0), f20(0.0, 0.0, 0.0, 0.0, 0.0),
          i10(5, 0) + f20(0.5, 0.0) + i10(1, 0),
          "/PART/1", "block", i10(1, 1, 0), "/PART/2", "strip", i10(2, 2, 0),
          "/BRICK/1"]
    L += [i10(k + 1, *(cb[k] + 1)) for k in range(cb.shape[0])]
    L += ["/SHELL/2"]
    L += [i10(100 + k, *(cs[k] + 1)) for k in range(cs.shape[0])]
    L += ["/SKEW/FIX/7", "rotated", f20(0, 0, 0), f20(0.0, 0.8, 0.6), f20(0.0, -0.6, 0.8)]
    base = [k + 1 for k in range(xb.shape[0]) if xb[k, 2] == 0.0]
    L += ["/BCS/1", "base", "   001 000" + i10(7, 1), "/GRNOD/NODE/1", "base"]
    L += [i10(*base[i:i + 10]) for i in range(0, len(base), 10)]
    edge = [xb.shape[0] + k + 1 for k in range(xs.shape[0]) if xs[k, 0] == 5.0]
    L += ["/BCS/2", "edge", "   111 111" + i10(0, 2), "/GRNOD/NODE/2", "edge"]
    L += [i10(*edge[i:i + 10]) for i in range(0, len(edge), 10)]
    L += ["/FUNCT/11", "ramp", f20(0.0, 0.0), f20(1e-6, 1.0), f20(1.0, 1.0),
          "/FUNCT/12", "constant", f20(0.0, 1.0)]
    top = cb[np.isclose(xb[cb[:, 4], 2], 3.0)][:, 4:8] + 1
    L += ["/SURF/SEG/21", "top"] + [i10(k + 1, *top[k]) for k in range(top.shape[0])]
    L += ["/SURF/PART/22", "strip", i10(2)]
    L += ["/PLOAD/31", "top pressure", i10(21, 11, 0, 0) + " " * 20 + f20(1.0, -50.0),
          "/PLOAD/32", "strip pressure", i10(22, 12, 0, 0) + " " * 20 + f20(0.0, 2.0)]
    L += ["/CLOAD/41", "corner", i10(11) + "         Y" + i10(7, 0, 3, 0) + f20(1.0, 5.0),
          "/GRNOD/NODE/3", "corner", i10(xb.shape[0])]
    L += ["/TH/NODE/1", "output", "DEF", i10(1, 0), "/END"]
    open(path, "w").write("\n".join(L) + "\n")
    return xb, cb, xs, cs, top - 1, base, edge


def direct_deck(xb, cb, xs, cs, top, base, edge):
    x = np.vstack([xb, xs])
    p = decks.new_part(x)
    decks.add_hex(p, cb, decks.material(decks.LAW_ELASTIC, RHO, E, NU), decks.solid_prop())
    jc = decks.material(decks.LAW_JOHNSON_COOK, RHO, E, NU, 350.0, 275.0, 0.36)
    decks.add_shell(p, cs, jc, decks.shell_prop(0.5, npt=5, ithk=1))
    b = np.array(base) - 1
    p["icodt"][b] |= 1
    p["iskew"] = -np.ones(x.shape[0], np.int32)
    p["iskew"][b] = 0
    e = np.array(edge) - 1
    p["icodt"][e] |= 7
    p["icodr"][e] |= 7
    p["ploads"] = [dict(seg=top, func=0, ascale_x=1.0, fscale=-50.0),
                   dict(seg=cs, func=1, ascale_x=1.0, fscale=2.0)]
    p["cloads"] = [dict(nodes=np.array([xb.shape[0] - 1]), dir=2, skew=0, func=0, ascale_x=1.0, fscale=5.0)]
    d = decks.deck([p])
    d["functions"] = [dict(x=[0.0, 1e-6, 1.0], y=[0.0, 1.0, 1.0]), dict(x=[0.0], y=[1.0])]
    y, z = np.array([0.0, 0.8, 0.6]), np.array([0.0, -0.6, 0.8])
    xa = np.cross(y, z)
    d["skews"] = [np.concatenate([xa / np.linalg.norm(xa), np.cross(z, xa), z])]
    return d


def test_reader_builds_the_direct_deck_and_runs_alike(tmp_path):
    from oracle.oracle import Oracle
    path = tmp_path / "READ_0000.rad"
    parts = write_deck(path)
    got = rad.to_deck(rad.StarterDeck(str(path)))
    want = direct_deck(*parts)
    pg, pw = got["parts"][0], want["parts"][0]
    assert np.allclose(pg["ms"], pw["ms"], rtol=1e-12, atol=0)
    assert np.allclose(pg["inr"], pw["inr"], rtol=1e-12, atol=0)
    assert (pg["icodt"] == pw["icodt"]).all() and (pg["icodr"] == pw["icodr"]).all()
    assert (pg["iskew"] == pw["iskew"]).all()
    assert np.allclose(got["skews"][0], want["skews"][0], atol=1e-15)
    assert pg["hex"][0]["prop"] == pw["hex"][0]["prop"]
    assert pg["shell"][0]["prop"] == pw["shell"][0]["prop"]
    for a, b in zip(pg["ploads"], pw["ploads"]):
        assert (a["seg"] == b["seg"]).all() and a["fscale"] == b["fscale"] and a["func"] == b["func"]
    og, ow = Oracle(got), Oracle(want)
    og.step(80)
    ow.step(80)
    assert np.array_equal(og.get_nodes()["d"], ow.get_nodes()["d"])
    assert og.energies() == ow.energies()
    assert og.energies()["external_work"] != 0.0
    t = og.time()
    assert rad.element_id(got, t["ityptst"], t["neltst"]) is not None


def test_reader_refuses_what_it_does_not_implement(tmp_path):
    path = tmp_path / "BAD_0000.rad"
    write_deck(path)
    text = open(path).read().replace("/END", "/INTER/TYPE7/1\ncontact\n/END")
    open(path, "w").write(text)
    with pytest.raises(rad.RadError, match="INTER"):
        rad.StarterDeck(str(path))


@pytest.mark.parametrize("ishell,npt,hm,hr", [(2, 5, 0.01, 0.01), (3, 5, 0.1, 0.01), (4, 1, 0.01, 0.01)])
def test_reader_shell_formulations_and_their_defaults(tmp_path, ishell, npt, hm, hr):
    """Ishell 2 to 4 pass through with the starter's hourglass defaults (0.1, 0.1,
    0.01 for Ishell 3; hm_read_prop01.F:204-212) and Dn; other Ishell values are
    refused."""
    path = tmp_path / "FORM_0000.rad"
    write_deck(path)
    text = open(path).read()
    old = "/PROP/SHELL/2\nshell\n" + i10(0, 0, 0, 0) + " " * 20 + f20(0.0) + "\n" + f20(0.0, 0.0, 0.0, 0.0, 0.0) + \
        "\n" + i10(5, 0)
    assert old in text
    new = "/PROP/SHELL/2\nshell\n" + i10(ishell, 0, 0, 0) + " " * 20 + f20(0.0) + "\n" + \
        f20(0.0, 0.0, 0.0, 0.0, 0.02) + "\n" + i10(npt, 0)
    open(path, "w").write(text.replace(old, new))
    pr = rad.to_deck(rad.StarterDeck(str(path)))["parts"][0]["shell"][0]["prop"]
    assert pr["ishell"] == ishell and pr["npt"] == npt
    assert (pr["hm"], pr["hf"], pr["hr"]) == (hm, hm, hr)
    assert pr["dn"] == 0.02
    open(path, "w").write(text.replace(old, new.replace(i10(ishell, 0, 0, 0), i10(12, 0, 0, 0))))
    with pytest.raises(rad.RadError, match="Ishell 12"):
        rad.to_deck(rad.StarterDeck(str(path)))
