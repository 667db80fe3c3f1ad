"""Synthetic decks for the element cycle (numpy, seeded).

A deck is a plain dict of numpy arrays in the reference's layouts, handed to
both the product C-ABI (``openradioss_b200.ecycle``) and the CPU oracle:

* ``parts``: list of parts; each part holds its nodes
  ``x, v, vr`` (numnod, 3) float64, ``ms, inr`` (numnod,) float64,
  ``icodt, icodr`` (numnod,) int32 (/BCS 3-bit codes: 4 = x, 2 = y, 1 = z),
  and its groups ``hex`` / ``shell`` (lists of dicts with ``ixs`` (nel, 11) or
  ``ixc`` (nel, 7) int32, 1-based node numbers as in IXS/IXC, ``mat``,
  ``prop`` dicts and optional per-element ``vol0`` / ``thke``).

Starter semantics reproduced here (the starter itself is not on the path):

* hexa nodal mass rho0 * V0 / 8 per node, V0 from the 1-point Jacobian
  (starter/source/elements/solid/solide/smass3.F:79-94);
* shell nodal mass rho * thk * A / 4 and rotational inertia
  EMS * (A / 9 + thk^2 / 12) per node, IHBE < 11
  (starter/source/elements/shell/coque/cinmas.F:703, 1296);
* defaults qa = 1.1, qb = 0.05 (hm_read_prop14.F:348-349), qh = 0.1
  (hm_read_prop14.F:358-361), shell hm = hf = hr = 0.01 for Ishell = 1
  (hm_read_prop01.F:204-211), shear factor 5/6 (hm_read_prop01.F:228);
* LAW2 moduli G = E / 2(1+nu), K = E / 3(1-2nu), A11 = E/(1-nu^2),
  A12 = nu A11, shell sound speed sqrt(E/rho) (hm_read_mat02_jc.F90).
"""
from __future__ import annotations

import math

import numpy as np

# ---------------------------------------------------------------------------
# materials and properties
# ---------------------------------------------------------------------------

LAW_ELASTIC = 1
LAW_JOHNSON_COOK = 2


def material(law, rho, young, nu, jc_a=0.0, jc_b=0.0, jc_n=1.0, epsmax=1e20, sigmax=1e20):
    g = young / (2.0 * (1.0 + nu))
    bulk = young / (3.0 * (1.0 - 2.0 * nu))
    a11 = young / (1.0 - nu * nu)
    return dict(law=law, rho0=rho, young=young, nu=nu, shear=g, bulk=bulk, a11=a11,
                a12=nu * a11, ssp_shell=math.sqrt(young / rho), jc_a=jc_a, jc_b=jc_b,
                jc_n=(jc_n if jc_n != 0.0 else 1.0), epsmax=epsmax, sigmax=sigmax)


def steel_elastic():
    return material(LAW_ELASTIC, 7850.0, 210e9, 0.3)


def steel_jc():
    return material(LAW_JOHNSON_COOK, 7850.0, 210e9, 0.3, 350e6, 275e6, 0.36)


def aluminium_jc():
    return material(LAW_JOHNSON_COOK, 2700.0, 70e9, 0.33, 350e6, 275e6, 0.36)


def solid_prop(qa=1.1, qb=0.05, qh=0.1, jcvt=0):
    return dict(qa=qa, qb=qb, qh=qh, jcvt=jcvt)


def shell_prop(thk, npt=5, ithk=1, hm=0.01, hf=0.01, hr=0.01, shf=5.0 / 6.0, pressure=0.0, ishfram=0, ipla=0,
               ishell=1, dn=0.0):
    """/PROP/SHELL values; ipla is M2CPLR's return (0 radial, 1 Newton, 2 projection),
    ishell the formulation (1..4, as the starter leaves it), dn the one-point
    V-shape hourglass coefficient."""
    return dict(thk=thk, npt=npt, ithk=ithk, ipla=ipla, ishfram=ishfram, hm=hm, hf=hf, hr=hr, shf=shf,
                pressure=pressure, ishell=ishell, dn=dn)


# ---------------------------------------------------------------------------
# meshes
# ---------------------------------------------------------------------------

def hex_block(nx, ny, nz, h, origin=(0.0, 0.0, 0.0)):
    """Structured block of nx*ny*nz cubes of edge h.  Returns (x, conn) with
    0-based connectivity in the hexa numbering 1-4 bottom, 5-8 top,
    counter-clockwise, which gives a positive SDERI3 Jacobian."""
    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    # node id = i + (nx+1)*(j + (ny+1)*k)   (x fastest)
    nid = lambda i, j, k: i + (nx + 1) * (j + (ny + 1) * k)
    x = np.empty(((nx + 1) * (ny + 1) * (nz + 1), 3))
    x[nid(ii, jj, kk).ravel(), 0] = origin[0] + h * ii.ravel()
    x[nid(ii, jj, kk).ravel(), 1] = origin[1] + h * jj.ravel()
    x[nid(ii, jj, kk).ravel(), 2] = origin[2] + h * kk.ravel()
    ei, ej, ek = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ei, ej, ek = (a.transpose(2, 1, 0).ravel() for a in (ei, ej, ek))  # element order: x fastest
    conn = np.stack([nid(ei, ej, ek), nid(ei + 1, ej, ek), nid(ei + 1, ej + 1, ek), nid(ei, ej + 1, ek),
                     nid(ei, ej, ek + 1), nid(ei + 1, ej, ek + 1), nid(ei + 1, ej + 1, ek + 1),
                     nid(ei, ej + 1, ek + 1)], axis=1).astype(np.int64)
    return x, conn


def quad_plate(n, size, jitter=0.0, seed=0):
    """Square plate of n*n quads in the z=0 plane, counter-clockwise (normal +z);
    interior nodes jittered in-plane by U(-jitter, +jitter) * h."""
    h = size / n
    i, j = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="xy")
    x = np.zeros(((n + 1) * (n + 1), 3))
    x[:, 0] = (i * h).ravel()
    x[:, 1] = (j * h).ravel()
    if jitter > 0.0:
        rng = np.random.Generator(np.random.PCG64(seed))
        interior = ((i > 0) & (i < n) & (j > 0) & (j < n)).ravel()
        d = rng.uniform(-jitter * h, jitter * h, size=(interior.sum(), 2))
        x[interior, 0:2] += d
    nid = lambda a, b: a + (n + 1) * b
    ei, ej = np.meshgrid(np.arange(n), np.arange(n), indexing="xy")
    ei, ej = ei.ravel(), ej.ravel()
    conn = np.stack([nid(ei, ej), nid(ei + 1, ej), nid(ei + 1, ej + 1), nid(ei, ej + 1)], axis=1)
    edge = ((i == 0) | (i == n) | (j == 0) | (j == n)).ravel()
    return x, conn.astype(np.int64), edge


def hex_volumes(x, conn):
    """1-point Jacobian volume (sderi3.F:103-149)."""
    X = x[conn]  # (nel, 8, 3)
    d17 = X[:, 6] - X[:, 0]
    d28 = X[:, 7] - X[:, 1]
    d35 = X[:, 4] - X[:, 2]
    d46 = X[:, 5] - X[:, 3]
    j1 = d17 + d28 - d35 - d46
    j4 = d17 + d46 + d28 + d35
    j7 = d17 + d46 - d28 - d35
    return np.einsum("ij,ij->i", j1, np.cross(j4, j7)) / 64.0


def shell_areas(x, conn):
    X = x[conn]
    n = np.cross(X[:, 2] - X[:, 0], X[:, 3] - X[:, 1])
    return 0.5 * np.linalg.norm(n, axis=1)


def ixs_from_conn(conn):
    nel = conn.shape[0]
    ixs = np.zeros((nel, 11), dtype=np.int32)
    ixs[:, 0] = 1
    ixs[:, 1:9] = conn + 1
    ixs[:, 9] = 1
    ixs[:, 10] = np.arange(1, nel + 1)
    return ixs


def ixc_from_conn(conn):
    nel = conn.shape[0]
    ixc = np.zeros((nel, 7), dtype=np.int32)
    ixc[:, 0] = 1
    ixc[:, 1:5] = conn + 1
    ixc[:, 5] = 1
    ixc[:, 6] = np.arange(1, nel + 1)
    return ixc


# ---------------------------------------------------------------------------
# parts
# ---------------------------------------------------------------------------

def new_part(x):
    n = x.shape[0]
    return dict(x=np.ascontiguousarray(x, dtype=np.float64), v=np.zeros((n, 3)), vr=np.zeros((n, 3)),
                ms=np.zeros(n), inr=np.zeros(n), icodt=np.zeros(n, np.int32),
                icodr=np.zeros(n, np.int32), hex=[], shell=[])


def add_hex(part, conn, mat, prop):
    vol0 = hex_volumes(part["x"], conn)
    np.add.at(part["ms"], conn.ravel(), np.repeat(mat["rho0"] * vol0 / 8.0, 8))
    part["hex"].append(dict(ixs=ixs_from_conn(conn), mat=mat, prop=prop, vol0=vol0))


def add_shell(part, conn, mat, prop, thke=None):
    area = shell_areas(part["x"], conn)
    thk = np.full(conn.shape[0], prop["thk"]) if thke is None else np.asarray(thke, np.float64)
    ems = mat["rho0"] * thk * area / 4.0
    xi = ems * (area / 9.0 + thk * thk / 12.0)
    np.add.at(part["ms"], conn.ravel(), np.repeat(ems, 4))
    np.add.at(part["inr"], conn.ravel(), np.repeat(xi, 4))
    part["shell"].append(dict(ixc=ixc_from_conn(conn), mat=mat, prop=prop, thke=thk))


def deck(parts, dtfac_solid=0.9, dtfac_shell=0.9, ncycles=100, name="deck"):
    return dict(parts=parts, dtfac_solid=dtfac_solid, dtfac_shell=dtfac_shell, dtmx=1e20,
                ncycles=ncycles, name=name)


def num_elements(d):
    return sum(g["ixs"].shape[0] for p in d["parts"] for g in p["hex"]) + \
        sum(g["ixc"].shape[0] for p in d["parts"] for g in p["shell"])


def num_nodes(d):
    return sum(p["x"].shape[0] for p in d["parts"])


# ---------------------------------------------------------------------------
# the five workloads
# ---------------------------------------------------------------------------

def c1_hex_block(nx=10, ny=10, nz=40, h=1e-3, ncycles=1000, law=LAW_ELASTIC, vz=-10.0):
    """Plain FP64 hex block: nx*ny*nz 1 mm cubes, LAW1 steel, qh = 0.1, z = 0
    face clamped, all other nodes at vz m/s along z, DTFAC 0.9."""
    x, conn = hex_block(nx, ny, nz, h)
    p = new_part(x)
    add_hex(p, conn, steel_elastic() if law == LAW_ELASTIC else steel_jc(), solid_prop())
    base = np.isclose(x[:, 2], 0.0)
    p["icodt"][base] = 7
    p["v"][~base, 2] = vz
    return deck([p], ncycles=ncycles, name=f"hex_block_{nx}x{ny}x{nz}")


def c2_shell_plate(n=200, size=0.2, thk=1e-3, npt=5, pressure=2e6, ncycles=2000, seed=0,
                   jc_a=None, thke=None, law=LAW_JOHNSON_COOK, ipla=0, ishell=1, jitter=0.05):
    """Split-precision shell plate: n*n BT shells on a square plate, interior
    nodes jittered +-5 % of h, LAW2 aluminium, simply supported edges (z fixed),
    uniform pressure step; ishell picks the formulation (Ishell 1..4)."""
    x, conn, edge = quad_plate(n, size, jitter=jitter, seed=seed)
    p = new_part(x)
    mat = aluminium_jc() if law == LAW_JOHNSON_COOK else material(LAW_ELASTIC, 2700.0, 70e9, 0.33)
    hm = 0.1 if ishell == 3 else 0.01             # the starter's defaults (hm_read_prop01.F:204-212)
    add_shell(p, conn, mat, shell_prop(thk, npt=npt, pressure=pressure, ipla=ipla, ishell=ishell, hm=hm, hf=hm),
              thke=thke)
    if jc_a is not None:
        p["shell"][0]["jc_a"] = np.asarray(jc_a, np.float64)
    p["icodt"][edge] = 1
    return deck([p], ncycles=ncycles, name=f"shell_plate_{n}x{n}")


def c3_batched_parts(nparts=64, seed=0, ncycles=500, scale=1.0):
    """Batched uneven parts: per part hex block or BT plate (50/50), element
    count log-uniform in [1e3, 2e5] (times ``scale``), LAW1 or LAW2, initial
    velocity U(1, 20) m/s along a random direction (hex) or the normal (shell)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    parts = []
    for _ in range(nparts):
        is_hex = rng.random() < 0.5
        nel = int(round(math.exp(rng.uniform(math.log(1e3), math.log(2e5))) * scale))
        law = LAW_ELASTIC if rng.random() < 0.5 else LAW_JOHNSON_COOK
        vmag = rng.uniform(1.0, 20.0)
        if is_hex:
            # at least 3 elements across: a 1-element-wide column of 1-point hexas is
            # unstable at the element time step (its volumetric mode, omega^2 = 12 K / rho h^2,
            # is above the Courant estimate of sdlen3.F / mqviscb.F)
            nx = max(3, int(round((nel / 4.0) ** (1.0 / 3.0))))
            x, conn = hex_block(nx, nx, 4 * nx, 1e-3)
            p = new_part(x)
            add_hex(p, conn, steel_elastic() if law == LAW_ELASTIC else steel_jc(), solid_prop())
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            base = np.isclose(x[:, 2], 0.0)
            p["icodt"][base] = 7
            p["v"][~base] = vmag * d
        else:
            n = max(4, int(round(math.sqrt(nel))))
            x, conn, edge = quad_plate(n, n * 1e-3, jitter=0.05, seed=int(rng.integers(1 << 30)))
            p = new_part(x)
            mat = aluminium_jc() if law == LAW_JOHNSON_COOK else material(LAW_ELASTIC, 2700.0, 70e9, 0.33)
            add_shell(p, conn, mat, shell_prop(1e-3))
            p["icodt"][edge] = 1
            p["v"][~edge, 2] = vmag
        parts.append(p)
    return deck(parts, ncycles=ncycles, name=f"batched_{nparts}_parts_seed{seed}")


def c4_mixed_mesh(nx=100, ny=100, nz=200, h=1e-3, ncycles=5000, vz=-20.0, skin=True):
    """Large mixed mesh: nx*ny*nz LAW2 steel hexas with a 1 mm BT shell skin on
    the four lateral faces sharing the block's nodes; z = 0 clamped, vz m/s."""
    x, conn = hex_block(nx, ny, nz, h)
    p = new_part(x)
    add_hex(p, conn, steel_jc(), solid_prop())
    if skin:
        nid = lambda i, j, k: i + (nx + 1) * (j + (ny + 1) * k)
        quads = []
        k = np.arange(nz)
        for face in range(4):
            if face == 0:   # y = 0, outward normal -y
                a = np.arange(nx)
                A, K = np.meshgrid(a, k, indexing="xy")
                q = [nid(A, 0, K), nid(A, 0, K + 1), nid(A + 1, 0, K + 1), nid(A + 1, 0, K)]
            elif face == 1:  # x = nx, outward +x
                a = np.arange(ny)
                A, K = np.meshgrid(a, k, indexing="xy")
                q = [nid(nx, A, K), nid(nx, A, K + 1), nid(nx, A + 1, K + 1), nid(nx, A + 1, K)][::-1]
            elif face == 2:  # y = ny, outward +y
                a = np.arange(nx)
                A, K = np.meshgrid(a, k, indexing="xy")
                q = [nid(A, ny, K), nid(A + 1, ny, K), nid(A + 1, ny, K + 1), nid(A, ny, K + 1)]
            else:            # x = 0, outward -x
                a = np.arange(ny)
                A, K = np.meshgrid(a, k, indexing="xy")
                q = [nid(0, A, K), nid(0, A, K + 1), nid(0, A + 1, K + 1), nid(0, A + 1, K)]
            quads.append(np.stack([c.ravel() for c in q], axis=1))
        add_shell(p, np.concatenate(quads).astype(np.int64), steel_jc(), shell_prop(1e-3))
    base = np.isclose(x[:, 2], 0.0)
    p["icodt"][base] = 7
    p["icodr"][base] = 7
    p["v"][~base, 2] = vz
    return deck([p], ncycles=ncycles, name=f"mixed_{nx}x{ny}x{nz}")


def c5_adjoint_plate(n=200, ncycles=500, seed=1, **kw):
    """Adjoint workload: the shell plate with per-element yield stress
    A ~ U(300, 400) MPa and thickness ~ U(0.9, 1.1) mm."""
    rng = np.random.Generator(np.random.PCG64(seed))
    nel = n * n
    jc_a = rng.uniform(300e6, 400e6, nel)
    thke = rng.uniform(0.9e-3, 1.1e-3, nel)
    return c2_shell_plate(n=n, ncycles=ncycles, jc_a=jc_a, thke=thke, **kw)


def hat_rail(length=0.3, wall=0.03, top=0.05, h=5e-3, kink=(0.1, 0.2), offset=0.03, thk=1.5e-3,
             mass=500.0, v0=10.0, npt=3, sigmax=600e6, ncycles=400):
    """Crash rail: a hat section (two walls of height ``wall`` joined by a top
    of width ``top``) swept along x over ``length``, the section moving by
    ``offset`` along y on a linear S-ramp between x = kink[0] and kink[1]; BT
    shells of edge ~h, LAW2 steel with a yield cap, 3 integration points,
    /SHFRA/V4 element frames (ISHFRAM 2).  The end x = 0 is one rigid link
    (x, y, z) carrying an added ``mass`` at its first node, all its nodes
    starting at v0 along x; the end x = length is held along x; free wall
    edges and both ends are held along z, with the rotations of the ends and
    the x/y rotations of the wall edges fixed."""
    nw, nt = int(round(wall / h)), int(round(top / h))
    nc = int(round(length / h))
    # section rows: wall 1 at y = top (z up), top at z = wall, wall 2 at y = 0 (z down)
    rows = [(top, wall * k / nw) for k in range(nw)] + \
           [(top - top * k / nt, wall) for k in range(nt)] + \
           [(0.0, wall - wall * k / nw) for k in range(nw + 1)]
    nr = len(rows) - 1
    xc = np.linspace(0.0, length, nc + 1)
    ramp = offset * np.clip((xc - kink[0]) / (kink[1] - kink[0]), 0.0, 1.0)
    x = np.zeros(((nr + 1) * (nc + 1), 3))
    nid = lambda r, c: r * (nc + 1) + c
    for r, (y0, z) in enumerate(rows):
        x[nid(r, 0):nid(r, nc) + 1, 0] = xc
        x[nid(r, 0):nid(r, nc) + 1, 1] = y0 - ramp
        x[nid(r, 0):nid(r, nc) + 1, 2] = z
    R, Cc = np.meshgrid(np.arange(nr), np.arange(nc), indexing="ij")
    R, Cc = R.ravel(), Cc.ravel()
    conn = np.stack([nid(R, Cc), nid(R, Cc + 1), nid(R + 1, Cc + 1), nid(R + 1, Cc)], axis=1).astype(np.int64)
    p = new_part(x)
    mat = material(LAW_JOHNSON_COOK, 7850.0, 210e9, 0.3, 350e6, 275e6, 0.36, sigmax=sigmax)
    add_shell(p, conn, mat, shell_prop(thk, npt=npt, ithk=0, hr=1e-5, ishfram=2))
    left = np.array([nid(r, 0) for r in range(nr + 1)])
    right = np.array([nid(r, nc) for r in range(nr + 1)])
    edges = np.concatenate([np.arange(nid(0, 0), nid(0, nc) + 1), np.arange(nid(nr, 0), nid(nr, nc) + 1)])
    p["icodt"][edges] |= 1
    p["icodr"][edges] |= 6
    p["icodt"][left] |= 1
    p["icodr"][left] |= 7
    p["icodt"][right] |= 5
    p["icodr"][right] |= 7
    p["v"][left, 0] = v0
    p["ms"][left[0]] += mass
    p["rlinks"] = [dict(nodes=left, ic=7, icr=0)]
    return deck([p], ncycles=ncycles, name=f"hat_rail_{nr}x{nc}")
