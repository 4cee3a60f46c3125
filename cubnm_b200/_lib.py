"""Loads the in-tree CUDA library ``libcubnm_b200.so``.

There is no fallback: if the library is missing or cannot be loaded, importing
the simulation entry points raises, so a run can never silently fall back to
a CPU path.
"""
import ctypes as C
import os

from . import _abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcubnm_b200.so")
_LIB = None


def build():
    """Compiles the library in-tree (nvcc, sm_100a)."""
    import subprocess
    subprocess.run(["make", "-C", os.path.join(_HERE, "csrc"), "-s", "-j8"], check=True)


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"cubnm_b200: {LIB_PATH} is missing; build it with `make -C cubnm_b200/csrc` "
            "(or __graft_entry__.build()). There is no CPU fallback."
        )
    L = C.CDLL(LIB_PATH)
    _abi.declare(L, "cbnm_")
    L.cbnm_run_simulations_device.argtypes = [C.POINTER(_abi.RunArgs), C.POINTER(_abi.Outputs)]
    L.cbnm_run_simulations_device.restype = C.c_int
    L.cbnm_last_timing.argtypes = [C.POINTER(_abi.Timing)]
    L.cbnm_last_timing.restype = C.c_int
    L.cbnm_reset.argtypes = []
    L.cbnm_reset.restype = C.c_int
    dp = C.POINTER(C.c_double)
    L.cbnm_gof.argtypes = [dp, C.c_int, C.c_int, dp, dp, C.c_int, dp, C.c_int, dp, dp, dp, dp]
    L.cbnm_gof.restype = C.c_int
    _LIB = L
    return L


def check(status):
    if status != 0:
        raise RuntimeError(lib().cbnm_last_error().decode())
