"""The C ABI library loads and exports every symbol include/lym_b200.h declares
(no compute call: this runs without a GPU)."""
import ctypes
import os

import leonardym_b200 as L


def test_library_exports_every_declared_symbol():
    path = L._lib.LIB_PATH
    if not os.path.exists(path):
        L.build()
    so = ctypes.CDLL(path)
    names = L.declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing


def test_context_create_rejects_bad_geometry():
    lib = L.lib()
    ptr = ctypes.c_void_p()
    odd_t = (ctypes.c_int * 4)(4, 4, 4, 5)
    assert lib.lym_context_create(odd_t, 0, 0, ctypes.byref(ptr)) == -4
    bad_rep = (ctypes.c_int * 4)(4, 4, 4, 4)
    assert lib.lym_context_create(bad_rep, 7, 0, ctypes.byref(ptr)) == -1
    assert lib.lym_context_create(None, 0, 0, ctypes.byref(ptr)) == -1


def test_every_declared_symbol_has_a_typed_binding():
    # ctypes signatures for the whole C ABI: the context entry points in _lib.py, the
    # server's in server.py (without them ctypes would pass 64-bit values as int)
    here = os.path.dirname(L.__file__)
    src = "".join(open(os.path.join(here, f)).read() for f in ("_lib.py", "server.py"))
    untyped = [n for n in L.declared_symbols() if f'"{n}"' not in src and f"L.{n}.argtypes" not in src]
    assert not untyped, untyped
