"""Design sensitivities of the shell cycle: host helpers around or_ecycle_adjoint.

``ECycle.adjoint`` returns the partial derivatives the device computes: with
respect to each shell element's Johnson-Cook A, its thickness at the start of
the run, and the nodal masses and rotational inertias.  When the masses are
themselves functions of the thickness, as in the deck builder's lumping
(``decks.add_shell``: element mass rho*t*A/4 to each corner, inertia
m*(A/9 + t^2/12)), :func:`thickness_gradient` adds that chain so that the
result is dJ/dt of the deck as a function of its thicknesses.
"""
from __future__ import annotations

import numpy as np

from . import decks


def mass_chain(deck, dms, din):
    """Per shell group, sum_k dJ/dMS[n_k] dMS/dt + dJ/dIN[n_k] dIN/dt for each
    element, with the lumping of ``decks.add_shell``."""
    out = []
    for p, part in enumerate(deck["parts"]):
        for g in part["shell"]:
            conn = g["ixc"][:, 1:5] - 1
            area = decks.shell_areas(part["x"], conn)
            thk = np.asarray(g["thke"], np.float64)
            rho = g["mat"]["rho0"]
            ems = rho * thk * area / 4.0
            dems = rho * area / 4.0
            dxi = dems * (area / 9.0 + thk * thk / 12.0) + ems * thk / 6.0
            out.append(dms[p][conn].sum(axis=1) * dems + din[p][conn].sum(axis=1) * dxi)
    return out


def thickness_gradient(deck, res):
    """dJ/dt per shell group: the direct term plus the mass chain."""
    return [a + b for a, b in zip(res["dthk"], mass_chain(deck, res["dms"], res["din"]))]


def centre_node(deck, part=0):
    """Index of the node nearest to the centre of a part's bounding box."""
    x = deck["parts"][part]["x"]
    c = 0.5 * (x.min(axis=0) + x.max(axis=0))
    return int(np.argmin(((x - c) ** 2).sum(axis=1)))
