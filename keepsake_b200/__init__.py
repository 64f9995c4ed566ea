"""keepsake_b200: B200-native (sm_100a) small_pt path tracer behind a C ABI.

This Python module is a thin ctypes binding of ``libks_b200.so`` (declared in
``include/ks_b200.h``) used by the test-suite and ``bench.py``.  The library is the product;
there is no Python or CPU fallback: importing this module raises if the shared library has not
been built (``python -c "import __graft_entry__ as g; g.build()"`` or ``make -C keepsake_b200``).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libks_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"keepsake_b200: {LIB_PATH} is missing; build it with `make -C keepsake_b200` "
        "(the CUDA library is the only implementation)")

lib = ctypes.CDLL(LIB_PATH)

KS_OK = 0
STATUS_NAMES = {
    0: "KS_OK", 1: "KS_ERR_INVALID_ARGUMENT", 2: "KS_ERR_OUT_OF_MEMORY", 3: "KS_ERR_CUDA",
    4: "KS_ERR_QUEUE_OVERFLOW", 5: "KS_ERR_WATCHDOG", 6: "KS_ERR_NOT_BUILT",
    7: "KS_ERR_UNSUPPORTED", 8: "KS_ERR_PARSE", 9: "KS_ERR_IO",
}

_vp = ctypes.c_void_p
_u32 = ctypes.c_uint32
_i32 = ctypes.c_int32
_f32 = ctypes.c_float

lib.ks_context_create.argtypes = [ctypes.c_int, ctypes.POINTER(_vp)]
lib.ks_context_create.restype = ctypes.c_int
lib.ks_context_destroy.argtypes = [_vp]
lib.ks_context_destroy.restype = None
lib.ks_status_string.argtypes = [ctypes.c_int]
lib.ks_status_string.restype = ctypes.c_char_p
lib.ks_last_error.argtypes = [_vp]
lib.ks_last_error.restype = ctypes.c_char_p
lib.ks_sobol_points.argtypes = [_vp] + [_u32] * 11 + [_vp]
lib.ks_sobol_points.restype = ctypes.c_int


class KsError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{name}: {detail}" if detail else name)


def ptr(a) -> ctypes.c_void_p:
    """Address of a contiguous numpy array (or None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "arrays passed to the C ABI must be contiguous"
    return ctypes.c_void_p(a.ctypes.data)


class Context:
    """One CUDA device + stream (ks_context)."""

    def __init__(self, device: int = 0):
        h = _vp()
        st = lib.ks_context_create(device, ctypes.byref(h))
        if st != KS_OK:
            raise KsError(st, "ks_context_create")
        self.handle = h

    def check(self, st: int, what: str = ""):
        if st != KS_OK:
            raise KsError(st, f"{what}: {lib.ks_last_error(self.handle).decode()}")

    def close(self):
        if self.handle:
            lib.ks_context_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sobol_points(self, full_w, full_h, spp, seed, x0, y0, nx, ny, s0, ns, nd) -> np.ndarray:
        out = np.empty((ny, nx, ns, nd, 3), dtype=np.float32)
        st = lib.ks_sobol_points(self.handle, full_w, full_h, spp, seed, x0, y0, nx, ny, s0, ns, nd, ptr(out))
        self.check(st, "ks_sobol_points")
        return out
