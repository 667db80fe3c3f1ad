"""The allocation-free entry point against the regular one.

or_ecycle_hex_step_noalloc exists for callers that cannot let the library
allocate device memory (an engine that reserves one device pool at start-up
and keeps its footprint fixed through the time loop).  The caller owns every
array; the library's only scratch, the FSKY force skyline, is a static device
array.  Here the test itself allocates the arrays (with torch) and checks,
over two calls in a row, that the results match the handle-based
or_ecycle_step path at the FP64 parity bar used by the other GPU tests.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from openradioss_b200 import abi, decks

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


def reference_skyline(conn, numnod):
    """Parith/ON tables: slots of a node in ascending element order (the
    starter's CNE order), iads = slot of each element corner."""
    nel = conn.shape[0]
    counts = np.bincount(conn.ravel(), minlength=numnod)
    adsky = np.zeros(numnod + 1, np.int32)
    adsky[1:] = np.cumsum(counts)
    nxt = adsky[:-1].copy()
    iads = np.zeros((nel, 8), np.int32)
    for e in range(nel):
        for k in range(8):
            n = conn[e, k]
            iads[e, k] = nxt[n]
            nxt[n] += 1
    return iads, adsky


@pytest.mark.parametrize("law,vz", [(decks.LAW_ELASTIC, -10.0), (decks.LAW_JOHNSON_COOK, -60.0)])
def test_noalloc_matches_handle_two_calls(law, vz):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from openradioss_b200 import build
    from openradioss_b200.ecycle import ECycle, load_library
    build.build()
    lib = load_library()
    f = lib.or_ecycle_hex_step_noalloc
    P, dp, ip = C.c_void_p, C.c_void_p, C.c_void_p
    f.argtypes = [C.c_int, P, C.c_int, C.POINTER(abi.Time), C.c_int, dp, dp, dp, dp, ip, C.c_int, ip, ip, ip,
                  C.POINTER(abi.Material), C.POINTER(abi.SolidProp), C.c_double, C.c_double, C.c_double,
                  dp, dp, dp, dp, dp, dp, dp]
    f.restype = C.c_int

    d = decks.c1_hex_block(nx=5, ny=4, nz=10, law=law, vz=vz)
    p = d["parts"][0]
    g = p["hex"][0]
    conn = (g["ixs"][:, 1:9] - 1).astype(np.int32)
    numnod, nel = p["x"].shape[0], conn.shape[0]
    iads, adsky = reference_skyline(conn, numnod)

    dev = torch.device("cuda", 0)
    t64 = lambda a: torch.tensor(np.ascontiguousarray(a, np.float64), device=dev)
    t32 = lambda a: torch.tensor(np.ascontiguousarray(a, np.int32), device=dev)
    X, D, V = t64(p["x"]), torch.zeros((numnod, 3), dtype=torch.float64, device=dev), t64(p["v"])
    MS, CODE = t64(p["ms"]), t32(p["icodt"])
    CONN, IADS, ADSKY = t32(conn), t32(iads), t32(adsky)
    SIG = torch.zeros((6, nel), dtype=torch.float64, device=dev)
    EINT, QVIS, PLA, EPSD = (torch.zeros(nel, dtype=torch.float64, device=dev) for _ in range(4))
    RHO = torch.full((nel,), g["mat"]["rho0"], dtype=torch.float64, device=dev)
    VOL0 = t64(g["vol0"])
    mat, prop = abi.make_material(g["mat"]), abi.make_solid_prop(g["prop"])
    t = abi.initial_time()
    stream = torch.cuda.current_stream().cuda_stream
    ptr = lambda a: C.c_void_p(a.data_ptr())

    h = ECycle(d, precision=abi.OR_PREC_FP64)
    for call in range(2):
        n = 45 if call == 0 else 38
        torch.cuda.synchronize()
        rc = f(0, C.c_void_p(stream), n, C.byref(t), numnod, ptr(X), ptr(D), ptr(V), ptr(MS), ptr(CODE), nel,
               ptr(CONN), ptr(IADS), ptr(ADSKY), C.byref(mat), C.byref(prop), 0.9, 1e20, abi.DT_GROWTH_REF,
               ptr(SIG), ptr(EINT), ptr(RHO), ptr(QVIS), ptr(PLA), ptr(EPSD), ptr(VOL0))
        assert rc == 0
        h.step(n)
        ref = h.get_nodes()
        st = h.hex_state(0)
        assert rel(D.cpu().numpy(), ref["d"]) < FP64_TOL
        assert rel(V.cpu().numpy(), ref["v"]) < FP64_TOL
        assert rel(SIG.cpu().numpy(), st["sig"]) < FP64_TOL
        assert rel(EINT.cpu().numpy(), st["eint"]) < FP64_TOL
        if law == decks.LAW_JOHNSON_COOK:
            assert rel(PLA.cpu().numpy(), st["pla"]) < FP64_TOL
        assert t.ncycle == h.time()["ncycle"]
        assert abs(t.dt2 - h.time()["dt2"]) <= FP64_TOL * h.time()["dt2"]
        assert abs(t.tt - h.time()["tt"]) <= FP64_TOL * h.time()["tt"]


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
    nel = abi_max = 262144 // 8 + 1
    rc = f(C.c_int(0), None, C.c_int(1), C.byref(t), C.c_int(8), dummy, dummy, dummy, dummy, dummy, C.c_int(nel),
           dummy, dummy, dummy, C.byref(mat), C.byref(prop), C.c_double(0.9), C.c_double(1e20), C.c_double(1.1),
           dummy, dummy, dummy, dummy, dummy, dummy, dummy)
    assert rc == abi.OR_E_ARG
    assert abi_max * 8 > 262144
