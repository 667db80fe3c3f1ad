"""The C-ABI library loads without a GPU and exports every entry point that
include/or_ecycle.h declares (no compute calls are made here)."""
import ctypes
import os
import re

from openradioss_b200 import build
from openradioss_b200.ecycle import EXPORTS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^\s*(?:int|const char\*)\s+(or_ecycle_\w+)\s*\(", src, re.M)
    return sorted(set(names))


def test_header_declares_the_binding_list():
    assert sorted(EXPORTS) == [n for n in declared_functions() if n in EXPORTS]
    assert set(EXPORTS) <= set(declared_functions())


def test_library_exports_every_declared_symbol():
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_create_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    from openradioss_b200 import abi
    lib = ctypes.CDLL(build.build())
    cfg = abi.make_config()
    h = ctypes.c_void_p()
    rc = lib.or_ecycle_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == abi.OR_E_CUDA and not h.value
