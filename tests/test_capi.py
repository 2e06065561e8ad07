"""CPU: the C-ABI library loads and exports every symbol include/*.h declares
(no compute calls without a GPU)."""
import ctypes
import glob
import os
import re

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(csffci_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_symbol():
    from pyscf_forge_b200 import _capi
    lib = _capi.load()
    declared = _declared()
    assert declared, "no declarations parsed"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    # every declared entry point has a ctypes signature in the binding
    assert declared <= set(_capi.exported_symbols()), sorted(declared - set(_capi.exported_symbols()))
    assert lib.csffci_abi_version() == 1


def test_struct_layouts():
    from pyscf_forge_b200 import _capi
    assert ctypes.sizeof(_capi.LinkEntry) == 8
    assert ctypes.sizeof(_capi.Block) == 64
