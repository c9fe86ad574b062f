"""Load the in-tree libchaoslab_b200.so. There is no fallback: a missing or unloadable library is an error."""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libchaoslab_b200.so")
_lock = threading.Lock()
_lib = None


class LibraryMissing(RuntimeError):
    pass


def lib() -> C.CDLL:
    """The loaded library (built by `chaos_b200.build.build()` / `__graft_entry__.build()`)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise LibraryMissing(f"{LIB_PATH} is not built; run __graft_entry__.build() first")
            _lib = _abi.declare(C.CDLL(LIB_PATH))
        return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().cl_b200_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def menu() -> list[str]:
    L = lib()
    return [L.cl_b200_menu_key(i).decode() for i in range(L.cl_b200_menu_size())]
