"""The allocation-free entry point against the regular one and the oracle.

or_ecycle_hex_step_noalloc exists for callers that cannot let the library
allocate device memory (an engine that reserves one device pool at start-up
and keeps its footprint fixed through the time loop).  The caller owns every
array; the library's only scratch, the FSKY force skyline, is a static device
array.  Here the test itself allocates the arrays (with torch) and checks,
over two calls in a row, that the results match the handle-based
or_ecycle_step path and the CPU oracle at the FP64 parity bar used by the
other GPU tests; that the largest group the scratch holds (32,768 hexas, every
slot used) runs; and that tables outside the scratch or not a permutation are
refused before anything is written.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from openradioss_b200 import abi, decks

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
MAX_SLOTS = 262144


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def reference_skyline(conn, numnod):
    """Parith/ON tables: slots of a node in ascending element order (the
    starter's CNE order), iads = slot of each element corner."""
    nel = conn.shape[0]
    counts = np.bincount(conn.ravel(), minlength=numnod)
    adsky = np.zeros(numnod + 1, np.int32)
    adsky[1:] = np.cumsum(counts)
    order = np.argsort(conn.ravel(), kind="stable")          # corners by node, then element
    iads = np.empty(8 * nel, np.int32)
    iads[order] = np.arange(8 * nel, dtype=np.int32)
    return iads.reshape(nel, 8), adsky


def entry():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openradioss_b200 import build
    from openradioss_b200.ecycle import load_library
    build.build()
    lib = load_library()
    f = lib.or_ecycle_hex_step_noalloc
    P = C.c_void_p
    f.argtypes = [C.c_int, P, C.c_int, C.POINTER(abi.Time), C.c_int, P, P, P, P, P, C.c_int, P, P, P,
                  C.POINTER(abi.Material), C.POINTER(abi.SolidProp), C.c_double, C.c_double, C.c_double,
                  P, P, P, P, P, P, P]
    f.restype = C.c_int
    return f


class Arrays:
    """Caller-owned device arrays of one hexa group (allocated by the caller, here torch)."""

    def __init__(self, d, iads=None, adsky=None):
        import torch
        p = d["parts"][0]
        g = p["hex"][0]
        conn = (g["ixs"][:, 1:9] - 1).astype(np.int32)
        self.numnod, self.nel = p["x"].shape[0], conn.shape[0]
        if iads is None:
            iads, adsky = reference_skyline(conn, self.numnod)
        dev = torch.device("cuda", 0)
        t64 = lambda a: torch.tensor(np.ascontiguousarray(a, np.float64), device=dev)
        t32 = lambda a: torch.tensor(np.ascontiguousarray(a, np.int32), device=dev)
        self.X, self.D, self.V = t64(p["x"]), torch.zeros((self.numnod, 3), dtype=torch.float64, device=dev), t64(p["v"])
        self.MS, self.CODE = t64(p["ms"]), t32(p["icodt"])
        self.CONN, self.IADS, self.ADSKY = t32(conn), t32(iads), t32(adsky)
        self.SIG = torch.zeros((6, self.nel), dtype=torch.float64, device=dev)
        self.EINT, self.QVIS, self.PLA, self.EPSD = (torch.zeros(self.nel, dtype=torch.float64, device=dev)
                                                     for _ in range(4))
        self.RHO = torch.full((self.nel,), g["mat"]["rho0"], dtype=torch.float64, device=dev)
        self.VOL0 = t64(g["vol0"])
        self.mat, self.prop = abi.make_material(g["mat"]), abi.make_solid_prop(g["prop"])
        self.t = abi.initial_time()

    def call(self, f, ncycles):
        import torch
        ptr = lambda a: C.c_void_p(a.data_ptr())
        stream = torch.cuda.current_stream().cuda_stream
        torch.cuda.synchronize()
        return f(0, C.c_void_p(stream), ncycles, C.byref(self.t), self.numnod, ptr(self.X), ptr(self.D),
                 ptr(self.V), ptr(self.MS), ptr(self.CODE), self.nel, ptr(self.CONN), ptr(self.IADS),
                 ptr(self.ADSKY), C.byref(self.mat), C.byref(self.prop), 0.9, 1e20, abi.DT_GROWTH_REF,
                 ptr(self.SIG), ptr(self.EINT), ptr(self.RHO), ptr(self.QVIS), ptr(self.PLA), ptr(self.EPSD),
                 ptr(self.VOL0))


def check_against_handle(a, h, law):
    ref = h.get_nodes()
    st = h.hex_state(0)
    assert rel(a.D.cpu().numpy(), ref["d"]) < FP64_TOL
    assert rel(a.V.cpu().numpy(), ref["v"]) < FP64_TOL
    assert rel(a.SIG.cpu().numpy(), st["sig"]) < FP64_TOL
    assert rel(a.EINT.cpu().numpy(), st["eint"]) < FP64_TOL
    if law == decks.LAW_JOHNSON_COOK:
        assert rel(a.PLA.cpu().numpy(), st["pla"]) < FP64_TOL
    ht = h.time()
    assert a.t.ncycle == ht["ncycle"]
    assert abs(a.t.dt2 - ht["dt2"]) <= FP64_TOL * ht["dt2"]
    assert abs(a.t.tt - ht["tt"]) <= FP64_TOL * ht["tt"]
    assert a.t.ityptst == ht["ityptst"] == 1
    assert a.t.neltst == ht["neltst"]


@pytest.mark.parametrize("law,vz", [(decks.LAW_ELASTIC, -10.0), (decks.LAW_JOHNSON_COOK, -60.0)])
def test_noalloc_matches_handle_and_oracle_two_calls(law, vz):
    from openradioss_b200.ecycle import ECycle
    from oracle.oracle import Oracle
    f = entry()
    d = decks.c1_hex_block(nx=5, ny=4, nz=10, law=law, vz=vz)
    a = Arrays(d)
    h = ECycle(d, precision=abi.OR_PREC_FP64)
    o = Oracle(d, nthreads=4)
    for n in (45, 38):
        assert a.call(f, n) == 0
        h.step(n)
        o.step(n)
        check_against_handle(a, h, law)
        orf = o.get_nodes()
        assert rel(a.D.cpu().numpy(), orf["d"]) < FP64_TOL
        assert rel(a.V.cpu().numpy(), orf["v"]) < FP64_TOL
        ost = o.hex_state(0)
        assert rel(a.SIG.cpu().numpy(), ost["sig"]) < FP64_TOL
        assert abs(a.t.dt2 - o.time()["dt2"]) <= FP64_TOL * o.time()["dt2"]


def test_noalloc_largest_group_every_slot():
    """32x32x32 hexas: 8 * 32,768 = 262,144 skyline slots, the whole scratch."""
    from openradioss_b200.ecycle import ECycle
    f = entry()
    d = decks.c1_hex_block(nx=32, ny=32, nz=32, law=decks.LAW_JOHNSON_COOK, vz=-60.0)
    a = Arrays(d)
    assert 8 * a.nel == MAX_SLOTS
    h = ECycle(d, precision=abi.OR_PREC_FP64)
    for n in (12, 9):
        assert a.call(f, n) == 0
        h.step(n)
        check_against_handle(a, h, decks.LAW_JOHNSON_COOK)


@pytest.mark.parametrize("fault", ["slot_beyond_scratch", "negative_slot", "duplicate_slot",
                                   "slot_of_other_node", "adsky_total"])
def test_noalloc_refuses_bad_tables(fault):
    """A table the scratch cannot honour returns OR_E_ARG before any cycle runs:
    the caller's arrays are left as they were, and neltst names the element (or
    node) at fault."""
    f = entry()
    d = decks.c1_hex_block(nx=3, ny=3, nz=4)
    conn = (d["parts"][0]["hex"][0]["ixs"][:, 1:9] - 1).astype(np.int32)
    numnod = d["parts"][0]["x"].shape[0]
    iads, adsky = reference_skyline(conn, numnod)
    iads = iads.copy()
    adsky = adsky.copy()
    bad_elem = 7
    if fault == "slot_beyond_scratch":
        iads[bad_elem, 3] = MAX_SLOTS + 5          # a global LSKY number past the scratch
    elif fault == "negative_slot":
        iads[bad_elem, 3] = -1
    elif fault == "duplicate_slot":
        n = int(np.argmax(np.diff(adsky)))          # a node shared by the most corners
        corners = np.nonzero(conn.ravel() == n)[0]
        k, k_first = int(corners[-1]), int(corners[0])
        iads.ravel()[k] = iads.ravel()[k_first]     # the node's first slot, taken twice
    elif fault == "slot_of_other_node":
        iads[bad_elem, 0], iads[bad_elem, 1] = iads[bad_elem, 1], iads[bad_elem, 0]
    elif fault == "adsky_total":
        adsky[-1] += 1
        bad_elem = numnod - 1
    a = Arrays(d, iads, adsky)
    x0, v0 = a.X.cpu().numpy().copy(), a.V.cpu().numpy().copy()
    rc = a.call(f, 5)
    assert rc == abi.OR_E_ARG
    assert a.t.ncycle == 0
    if fault == "duplicate_slot":
        assert a.t.neltst in (k // 8, k_first // 8)     # whichever corner came second
    else:
        assert a.t.neltst == bad_elem
    assert np.array_equal(a.X.cpu().numpy(), x0)
    assert np.array_equal(a.V.cpu().numpy(), v0)
    assert not a.D.cpu().numpy().any()
    assert not a.SIG.cpu().numpy().any()
    # the same arrays with good tables run afterwards: the scratch holds no stale state
    iads_ok, adsky_ok = reference_skyline(conn, numnod)
    a.IADS.copy_(__import__("torch").tensor(iads_ok))
    a.ADSKY.copy_(__import__("torch").tensor(adsky_ok))
    a.t = abi.initial_time()
    assert a.call(f, 5) == 0
    assert a.t.ncycle == 5


def test_noalloc_rejects_oversized_group():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openradioss_b200.ecycle import load_library
    lib = load_library()
    f = lib.or_ecycle_hex_step_noalloc
    f.restype = C.c_int
    dummy = C.c_void_p(16)            # never dereferenced: the size check comes first
    t = abi.initial_time()
    mat, prop = abi.make_material(decks.steel_elastic()), abi.make_solid_prop(decks.solid_prop())
    nel = MAX_SLOTS // 8 + 1
    rc = f(C.c_int(0), None, C.c_int(1), C.byref(t), C.c_int(8), dummy, dummy, dummy, dummy, dummy, C.c_int(nel),
           dummy, dummy, dummy, C.byref(mat), C.byref(prop), C.c_double(0.9), C.c_double(1e20), C.c_double(1.1),
           dummy, dummy, dummy, dummy, dummy, dummy, dummy)
    assert rc == abi.OR_E_ARG
