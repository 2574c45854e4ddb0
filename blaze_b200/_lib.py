"""Loads libblaze_b200.so (built in-tree) and binds its C ABI.

There is no fallback: if the library is missing or cannot be loaded the
import fails with the reason.
"""
import ctypes as C
import os

from . import _abi
from .build import LIB

_lib = None


class BlazeError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"blaze_b200 error {code}: {msg}")
        self.code = code


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise ImportError(f"{LIB} is missing: run `python -m blaze_b200.build` "
                              "(or __graft_entry__.build()) first")
        _lib = _abi.bind(C.CDLL(LIB))
    return _lib


def check(rc, handle=None):
    if rc != _abi.BLZ_OK:
        lib = load()
        msg = lib.blz_last_error(handle).decode(errors="replace")
        raise BlazeError(rc, msg)
    return rc
