"""The C-ABI library builds for sm_100a, loads without a GPU and exports every
entry point declared in include/*.h."""
import ctypes
import glob
import os
import re

from tests.helpers import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        names |= set(re.findall(r"^\s*(?:int|const char\*)\s+(psb_\w+)\s*\(", txt, flags=re.M))
    return names


def test_library_builds_and_exports_every_declared_symbol():
    from pyspectral_b200 import build, _capi
    path = build.build()
    lib = ctypes.CDLL(path)
    declared = _declared()
    assert len(declared) >= 15
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_capi.EXPORTS) == declared


def test_create_rejects_bad_sizes_without_a_gpu():
    from pyspectral_b200 import _capi, build
    lib = _capi.load(build.build())
    g = _capi.Grid(10, 16, 16, 6.28, 6.28, 6.28, 0.6, 0.4, 0.4, 5)
    h = ctypes.c_void_p()
    st = lib.psb_ctx_create(ctypes.byref(g), 64, 0, ctypes.byref(h))
    assert st != 0 and not h.value
    assert b"multiple" in lib.psb_create_error() or b"factor" in lib.psb_create_error()
    g = _capi.Grid(16, 16, 16, 6.28, 6.28, 6.28, 0.4, 0.4, 0.4, 8)
    assert lib.psb_ctx_create(ctypes.byref(g), 48, 0, ctypes.byref(h)) != 0
    assert lib.psb_rhs(None, 0, None, None, None, None, None, None) != 0
