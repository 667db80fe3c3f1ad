"""Synthetic decks: sizes of the five workloads and starter mass semantics."""
import numpy as np

from openradioss_b200 import decks


def test_c1_sizes_and_mass():
    d = decks.c1_hex_block()
    p = d["parts"][0]
    assert p["x"].shape[0] == 4961
    assert p["hex"][0]["ixs"].shape == (4000, 11)
    vol = p["hex"][0]["vol0"]
    np.testing.assert_allclose(vol, 1e-9, rtol=1e-12)
    np.testing.assert_allclose(p["ms"].sum(), 7850.0 * vol.sum(), rtol=1e-12)
    assert (p["icodt"] == 7).sum() == 121


def test_c2_sizes_and_jitter():
    d = decks.c2_shell_plate()
    p = d["parts"][0]
    assert p["x"].shape[0] == 40401
    assert p["shell"][0]["ixc"].shape == (40000, 7)
    area = decks.shell_areas(p["x"], p["shell"][0]["ixc"][:, 1:5] - 1)
    np.testing.assert_allclose(area.sum(), 0.04, rtol=1e-12)
    h = 0.2 / 200
    grid = np.stack(np.meshgrid(np.arange(201) * h, np.arange(201) * h, indexing="xy"), -1).reshape(-1, 2)
    assert np.abs(p["x"][:, :2] - grid).max() <= 0.05 * h + 1e-15
    np.testing.assert_allclose(p["ms"].sum(), 2700 * 1e-3 * 0.04, rtol=1e-12)


def test_c3_parts_log_uniform():
    d = decks.c3_batched_parts(nparts=64, seed=0)
    assert len(d["parts"]) == 64
    n = [decks.num_elements(dict(parts=[p])) for p in d["parts"]]
    assert min(n) >= 500 and max(n) <= 3e5


def test_c4_sizes():
    d = decks.c4_mixed_mesh(nx=10, ny=10, nz=20)
    p = d["parts"][0]
    assert p["hex"][0]["ixs"].shape[0] == 2000
    assert p["shell"][0]["ixc"].shape[0] == 4 * 10 * 20
    assert (p["hex"][0]["vol0"] > 0).all()


def test_c5_per_element_parameters():
    d = decks.c5_adjoint_plate(n=20)
    g = d["parts"][0]["shell"][0]
    assert g["jc_a"].min() >= 300e6 and g["jc_a"].max() <= 400e6
    assert g["thke"].min() >= 0.9e-3 and g["thke"].max() <= 1.1e-3
