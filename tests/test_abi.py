"""C-ABI boundary checks that need no GPU: the library loads, exports every entry point the
public header declares, and reports errors as status codes without a device."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            src = open(os.path.join(inc, fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            for m in re.finditer(r"\b(ks_[a-z0-9_]+)\s*\(", src):
                names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    import keepsake_b200 as ks
    syms = declared_symbols()
    assert len(syms) >= 5
    missing = [s for s in sorted(syms) if not hasattr(ks.lib, s)]
    assert not missing, f"declared in include/*.h but not exported: {missing}"


def test_status_strings():
    import keepsake_b200 as ks
    for code in range(10):
        assert ks.lib.ks_status_string(code)


def test_context_without_device_returns_status():
    import keepsake_b200 as ks
    import torch
    if torch.cuda.is_available():
        return
    h = ctypes.c_void_p()
    st = ks.lib.ks_context_create(0, ctypes.byref(h))
    assert st != 0 and not h.value
