"""Loader of the engine's shared library (built in-tree by crushrs_b200.build).

The library is the product: every GPU entry point lives in it. There is no
Python or CPU fallback; a missing or stale library is an error.
"""
import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcrush_b200.so")

_lib = None


class CrushError(RuntimeError):
    """A non-OK status from the C ABI, with the library's message."""

    def __init__(self, status, message):
        self.status = status
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")


def lib():
    """The loaded library (built on first use if absent)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build

            build.build_library()
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"crushrs_b200 native library missing: {LIB_PATH}")
        handle = C.CDLL(LIB_PATH, mode=C.RTLD_GLOBAL)
        abi.declare_scenario_api(handle)
        abi.declare_engine_api(handle)
        _lib = handle
    return _lib


def check(status, allow=(abi.CRUSH_OK,)):
    """Raise CrushError unless `status` is one of `allow`; returns status."""
    if status not in allow:
        raise CrushError(status, lib().crush_last_error().decode())
    return status
